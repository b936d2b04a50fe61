// libpsm_cuda.so: C ABI (include/psm.h) over the sm_100a migration kernels (psm_kernels.cuh).
#include <cuda_runtime.h>
#include <omp.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "psm.h"
#include "psm_adjoint.cuh"
#include "psm_kernels.cuh"
#include "psm_segy.cuh"
#include "psm_vrms.cuh"

namespace {

using psm::FwdParams;
using psm::Job;

constexpr size_t kMaxDynSmem = 232448;  // 227 KB per CTA on sm_100

// Trace stride in HBM: n_t rounded up to 8 samples so every trace starts 32 B aligned for
// the TMA bulk copies; the tail samples stay zero.
inline int trace_stride(int n_t) { return (n_t + 7) & ~7; }

// Ring stage capacity (samples): 48 KB a stage, and at least one whole trace so a stage
// always takes a window.
inline int stage_cap(int ns, int store = psm::kStoreF32) {
    return std::max(psm::kStageCapMin * 8 / psm::store_bytes(store), ns);
}

// Storage of a geometry's traces (psm_precision -> psm::kStore*).
inline int store_of(int precision) {
    return precision == PSM_BF16 ? psm::kStoreBF16
                                 : precision == PSM_F16 ? psm::kStoreF16 : psm::kStoreF32;
}

int max_inline_window(const std::vector<Job>& jobs) {
    int m = 1;
    for (const Job& j : jobs) m = std::max(m, j.i1 - j.i0);
    return m;
}

// Failure injection for tests of the error paths (set from PSM_FAULT by psm_create):
// the g_fail_alloc-th device allocation from then on fails as if the device were out of
// memory (-1: never).
std::atomic<int> g_fail_alloc{-1};

bool alloc_fault_due() {
    int n = g_fail_alloc.load();
    while (n > 0) {
        if (g_fail_alloc.compare_exchange_weak(n, n - 1)) return n == 1;
    }
    return false;
}

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    cudaError_t ensure(size_t n) {
        if (n <= bytes && p) return cudaSuccess;
        release();
        if (alloc_fault_due()) return cudaErrorMemoryAllocation;
        cudaError_t e = cudaMalloc(&p, n ? n : 16);
        if (e == cudaSuccess) bytes = n;
        return e;
    }
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

struct Status {
    int code = PSM_OK;
    std::string msg;
    int fail(int c, const std::string& m) {
        code = c;
        msg = m;
        return c;
    }
};

#define PSM_CUDA_TRY(st, call)                                                          \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return (st).fail(e_ == cudaErrorMemoryAllocation ? PSM_ERR_NOMEM : PSM_ERR_CUDA, \
                             std::string(#call) + ": " + cudaGetErrorString(e_));        \
    } while (0)

// Dynamic shared memory of a forward launch (0: too large for one CTA).
size_t fwd_smem(const FwdParams& P, int store = psm::kStoreF32) {
    const size_t b = psm::smem_layout(P.max_inl, P.stage_cap, psm::store_bytes(store)).total;
    return b <= kMaxDynSmem ? b : 0;
}

constexpr int kDefaultVariant = PSM_FWD_PAIRS_O3;

inline bool is_j16(int variant) {
    return variant == PSM_FWD_PACKED_G4_J16 || variant == PSM_FWD_SCALAR_G4_J16;
}

inline bool is_o3(int variant) {
    return variant == PSM_FWD_PACKED_G4_O3 || variant == PSM_FWD_SCALAR_G4_O3 ||
           variant == PSM_FWD_PAIRS_O3;
}

inline bool is_pairs(int variant) {
    return variant == PSM_FWD_PAIRS_O3 || variant == PSM_FWD_PAIRS;
}

// The variant that actually runs: 16-bit storage and compensated summation run the packed
// skip-4 kernel, with 16 blocks a lane (16-bit storage only: compensation's partial and
// compensation registers leave no room for 16), or built for 3 CTAs per SM, each with or
// without mirrored pairs.
inline int effective_variant(int variant, int store, bool kahan) {
    if (variant == PSM_FWD_DEFAULT) variant = kDefaultVariant;
    if (store == psm::kStoreF32 && !kahan) return variant;
    if (!kahan && is_j16(variant)) return PSM_FWD_PACKED_G4_J16;
    if (is_pairs(variant)) return variant;
    return is_o3(variant) ? PSM_FWD_PACKED_G4_O3 : PSM_FWD_PACKED_G4;
}

// One instantiation of the forward kernel templates (MINB: CTAs per SM the kernel is built
// for, 2 or 3).
template <bool AMP_, bool PACKED_, int GB_, int J_, int STORE_, bool KAHAN_, int MINB_ = 2,
          bool PAIRS_ = false>
struct KernelTag {
    static constexpr bool AMP = AMP_, PACKED = PACKED_, KAHAN = KAHAN_, PAIRS = PAIRS_;
    static constexpr int GB = GB_, J = J_, STORE = STORE_, MINB = MINB_;
};

// Samples per stage of the kernel built for 3 CTAs per SM (32 KB) or 4 (20 KB), so that its
// shared memory fits the SM three or four times.
inline int stage_cap_for(int minb, int store) {
    return psm::stage_bytes_for(minb) / psm::store_bytes(store);
}

template <class K>
auto grid_kernel() {
    if constexpr (K::MINB == 4)
        return psm::fwd_kernel_o4<K::AMP, K::PACKED, K::GB, K::J, K::STORE, K::KAHAN, K::PAIRS>;
    else if constexpr (K::MINB == 3)
        return psm::fwd_kernel_o3<K::AMP, K::PACKED, K::GB, K::J, K::STORE, K::KAHAN, K::PAIRS>;
    else
        return psm::fwd_kernel<K::AMP, K::PACKED, K::GB, K::J, K::STORE, K::KAHAN, K::PAIRS>;
}

// Calls f(KernelTag<...>{}) for the kernel that (amp, effective variant, store, kahan) names.
template <bool AMP, class F>
cudaError_t with_kernel_amp(int variant, int store, bool kahan, F&& f) {
    using psm::kStoreBF16;
    using psm::kStoreF16;
    using psm::kStoreF32;
    const bool j16 = is_j16(variant), o3 = is_o3(variant), pr = is_pairs(variant);
    // 16-bit storage or compensated summation with mirrored pairs
    if (pr && (store != kStoreF32 || kahan)) {
        switch (store * 2 + (kahan ? 1 : 0)) {
#define PSM_PAIR_CASE(ST, KA)                                                                \
    case ST * 2 + KA:                                                                        \
        return o3 ? f(KernelTag<AMP, true, 4, 8, ST, KA, 3, true>{})                         \
                  : f(KernelTag<AMP, true, 4, 8, ST, KA, 2, true>{});
            PSM_PAIR_CASE(kStoreF32, 1)
            PSM_PAIR_CASE(kStoreBF16, 0)
            PSM_PAIR_CASE(kStoreBF16, 1)
            PSM_PAIR_CASE(kStoreF16, 0)
            PSM_PAIR_CASE(kStoreF16, 1)
#undef PSM_PAIR_CASE
            default: return cudaErrorInvalidValue;
        }
    }
    switch (store * 2 + (kahan ? 1 : 0)) {
        case kStoreF32 * 2:
            switch (variant) {
                case PSM_FWD_SCALAR_G2: return f(KernelTag<AMP, false, 2, 8, kStoreF32, false>{});
                case PSM_FWD_SCALAR_G4: return f(KernelTag<AMP, false, 4, 8, kStoreF32, false>{});
                case PSM_FWD_PACKED_G2: return f(KernelTag<AMP, true, 2, 8, kStoreF32, false>{});
                case PSM_FWD_PACKED_G4: return f(KernelTag<AMP, true, 4, 8, kStoreF32, false>{});
                case PSM_FWD_PACKED_G4_J16:
                    return f(KernelTag<AMP, true, 4, 16, kStoreF32, false>{});
                case PSM_FWD_SCALAR_G4_J16:
                    return f(KernelTag<AMP, false, 4, 16, kStoreF32, false>{});
                case PSM_FWD_PACKED_G8: return f(KernelTag<AMP, true, 8, 8, kStoreF32, false>{});
                case PSM_FWD_SCALAR_G8: return f(KernelTag<AMP, false, 8, 8, kStoreF32, false>{});
                case PSM_FWD_PACKED_G4_O3:
                    return f(KernelTag<AMP, true, 4, 8, kStoreF32, false, 3>{});
                case PSM_FWD_SCALAR_G4_O3:
                    return f(KernelTag<AMP, false, 4, 8, kStoreF32, false, 3>{});
                case PSM_FWD_PAIRS_O3:
                    return f(KernelTag<AMP, true, 4, 8, kStoreF32, false, 3, true>{});
                case PSM_FWD_PAIRS: return f(KernelTag<AMP, true, 4, 8, kStoreF32, false, 2, true>{});
                case PSM_FWD_PAIRS_J4_O4:
                    return f(KernelTag<AMP, true, 4, 4, kStoreF32, false, 4, true>{});


                default: return cudaErrorInvalidValue;
            }
        case kStoreF32 * 2 + 1:
            return o3 ? f(KernelTag<AMP, true, 4, 8, kStoreF32, true, 3>{})
                      : f(KernelTag<AMP, true, 4, 8, kStoreF32, true>{});
        case kStoreBF16 * 2:
            return j16  ? f(KernelTag<AMP, true, 4, 16, kStoreBF16, false>{})
                   : o3 ? f(KernelTag<AMP, true, 4, 8, kStoreBF16, false, 3>{})
                        : f(KernelTag<AMP, true, 4, 8, kStoreBF16, false>{});
        case kStoreBF16 * 2 + 1:
            return o3 ? f(KernelTag<AMP, true, 4, 8, kStoreBF16, true, 3>{})
                      : f(KernelTag<AMP, true, 4, 8, kStoreBF16, true>{});
        case kStoreF16 * 2:
            return j16  ? f(KernelTag<AMP, true, 4, 16, kStoreF16, false>{})
                   : o3 ? f(KernelTag<AMP, true, 4, 8, kStoreF16, false, 3>{})
                        : f(KernelTag<AMP, true, 4, 8, kStoreF16, false>{});
        case kStoreF16 * 2 + 1:
            return o3 ? f(KernelTag<AMP, true, 4, 8, kStoreF16, true, 3>{})
                      : f(KernelTag<AMP, true, 4, 8, kStoreF16, true>{});
        default: return cudaErrorInvalidValue;
    }
}

template <class F>
cudaError_t with_kernel(bool amp, int variant, int store, bool kahan, F&& f) {
    variant = effective_variant(variant, store, kahan);
    return amp ? with_kernel_amp<true>(variant, store, kahan, f)
               : with_kernel_amp<false>(variant, store, kahan, f);
}

// The grid kernel's shared-memory limit, set before a stream capture (the attribute belongs
// to the kernel, so it must cover the largest launch of the capture).
template <class K>
cudaError_t prepare_grid(K, size_t smem) {
    return cudaFuncSetAttribute(grid_kernel<K>(), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(smem));
}

template <class K>
cudaError_t launch_grid(K, const FwdParams& P_in, int n_jobs, size_t smem, cudaStream_t s) {
    constexpr int TT = 32 * K::J;
    auto* kern = grid_kernel<K>();
    FwdParams P = P_in;
    if constexpr (K::MINB > 2) {  // smaller stages, so that MINB CTAs fit an SM
        P.stage_cap = std::max(stage_cap_for(K::MINB, K::STORE), P.ns);
        smem = std::min(smem, fwd_smem(P, K::STORE));
    }
    if (n_jobs > 65535) return cudaErrorInvalidValue;  // grid y
    dim3 grid((P.n_ox + psm::kTX - 1) / psm::kTX, n_jobs, (P.n_t + TT - 1) / TT);
    dim3 block(32 * (psm::kTX + 1));
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(s, &cap);
    if (e != cudaSuccess) return e;
    if (cap == cudaStreamCaptureStatusNone) {  // a capture was prepared by prepare_grid
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem));
        if (e != cudaSuccess) return e;
    }
    kern<<<grid, block, smem, s>>>(P);
    return cudaGetLastError();
}

// Launch the forward kernel for n_jobs jobs (P.max_inl and P.stage_cap set; P.pairs for fp32
// storage, P.words and P.scales for 16-bit storage).
cudaError_t launch_fwd(const FwdParams& P, int n_jobs, bool amp, int variant, cudaStream_t s,
                       int store = psm::kStoreF32, bool kahan = false) {
    if (n_jobs <= 0 || P.n_ox <= 0 || P.n_t <= 0) return cudaSuccess;
    const size_t smem = fwd_smem(P, store);
    if (!smem) return cudaErrorInvalidValue;
    return with_kernel(amp, variant, store, kahan,
                       [&](auto k) { return launch_grid(k, P, n_jobs, smem, s); });
}

// words[n_rows][ns] and scales[n_rows] from the fp32 rows (quantize_kernel, one warp a row).
cudaError_t quantize(const float* src, uint32_t* words, float* scales, size_t n_rows, int ns,
                     int store, cudaStream_t s) {
    if (!n_rows) return cudaSuccess;
    const unsigned blocks = static_cast<unsigned>(std::min<size_t>((n_rows + 7) / 8, 148 * 16));
    if (store == psm::kStoreBF16)
        psm::quantize_kernel<psm::kStoreBF16><<<blocks, 256, 0, s>>>(src, words, scales, n_rows, ns);
    else
        psm::quantize_kernel<psm::kStoreF16><<<blocks, 256, 0, s>>>(src, words, scales, n_rows, ns);
    return cudaGetLastError();
}

// pairs[n_rows][ns] from the fp32 rows (pair_kernel).
cudaError_t build_pairs(const float* src, float2* dst, size_t n_rows, int ns, cudaStream_t s) {
    if (!n_rows) return cudaSuccess;
    const size_t n = n_rows * static_cast<size_t>(ns);
    const unsigned blocks = static_cast<unsigned>(std::min<size_t>((n + 255) / 256, 148 * 64));
    psm::pair_kernel<<<blocks, 256, 0, s>>>(src, dst, n_rows, ns);
    return cudaGetLastError();
}

void fill_consts(FwdParams& P, float dt, float d_il, float d_xl, float tan2) {
    P.inv_dt = 1.0f / dt;  // migration_kernel.cpp:44
    P.idt2 = P.inv_dt * P.inv_dt;
    P.d_il = d_il;
    P.d_xl = d_xl;
    P.inv_dxl = 1.0f / d_xl;
    P.tan2 = tan2;
    P.tanth = std::sqrt(std::max(tan2, 0.0f));
    P.ntm1f = static_cast<float>(P.n_t) - 1.0f;
    P.ntm1m = std::nextafter(P.ntm1f, 0.0f);
    P.vs_x = P.n_t;  // dense Vrms cube [n_vrow][n_vx][n_t]
    P.vs_row = static_cast<long long>(P.n_vx) * P.n_t;
    P.pairable = 1;  // inline positions 0, 1, 2, ... (the per-inline drop-in checks its own)
}

// Argument checks of a geometry: PSM_OK, or the status with *why set.
int check_geometry(const psm_geom& g, std::string* why) {
    if (g.n_il <= 0 || g.n_xl <= 0 || g.n_t <= 0 || g.n_oi <= 0 || g.n_ox <= 0 || g.pad_il < 0 ||
        g.pad_xl < 0 || g.m_il < 0 || !(g.dt > 0.0f) || !(g.d_il > 0.0f) || !(g.d_xl > 0.0f) ||
        !(g.tan2_theta >= 0.0f)) {
        *why = "invalid geometry";
        return PSM_ERR_ARG;
    }
    if (g.precision != PSM_F32 && g.precision != PSM_BF16 && g.precision != PSM_F16) {
        *why = "precision must be PSM_F32, PSM_BF16 or PSM_F16";
        return PSM_ERR_ARG;
    }
    const int store = store_of(g.precision);
    const int ns = trace_stride(g.n_t);
    // inline window of any output inline <= 2 (m_il + pad_il) + 1 (+ the inline table) and one
    // whole trace per ring stage must fit the CTA's shared memory
    const int64_t win = std::min<int64_t>(g.n_il, 2 * (int64_t(g.m_il) + g.pad_il) + 1);
    if (psm::smem_layout(static_cast<int>(win), stage_cap(ns), 8).total > kMaxDynSmem ||
        psm::smem_layout(static_cast<int>(win), stage_cap(ns, store), psm::store_bytes(store))
                .total > kMaxDynSmem) {
        *why = "n_t / aperture too large for the staging ring";
        return PSM_ERR_UNSUPPORTED;
    }
    return PSM_OK;
}

// Jobs of a geometry: one per output inline (jobs_all, for term counts) and one per distinct
// migrated inline (jobs), the repeated output rows as (row, row it copies).  Padded output
// inlines migrate the nearest real inline (main.cpp:258-288); the buffer of real inline c is
// inlines [c - m_il - pad_il, c + m_il + 1 + pad_il) clamped to the cube
// (migration_kernel.cpp:404-409).  False when out_center names an inline outside the cube.
bool plan_jobs(const psm_geom& g, const int32_t* out_center, std::vector<Job>& jobs,
               std::vector<Job>& jobs_all, std::vector<std::pair<int, int>>& copies) {
    jobs.clear();
    jobs_all.clear();
    copies.clear();
    std::vector<int> first_row(g.n_il, -1);
    for (int o = 0; o < g.n_oi; ++o) {
        const int cc = out_center ? out_center[o] : std::min(std::max(o - g.pad_il, 0), g.n_il - 1);
        if (cc < 0 || cc >= g.n_il) return false;
        const int rs = std::max(0, cc - g.m_il), re = std::min(g.n_il, cc + g.m_il + 1);
        Job j;
        j.row = o;
        j.vrow = cc;
        j.pos = cc;
        j.i0 = std::max(0, rs - g.pad_il);
        j.i1 = std::min(g.n_il, re + g.pad_il);
        jobs_all.push_back(j);
        if (first_row[cc] < 0) {
            first_row[cc] = o;
            jobs.push_back(j);
        } else {
            copies.emplace_back(o, first_row[cc]);
        }
    }
    return true;
}

}  // namespace

// ---------------------------------------------------------------------------- context

namespace {

// Pinned staging for copies between pageable host memory and the device.  The CUDA driver
// copies pageable memory on one host thread through a small staging area of its own (about
// 11 GB/s here); these copies go through kStagingSlots pinned buffers that host threads
// (OpenMP) fill or drain in parallel, each buffer's device copy overlapping the host copy of
// the next.  Pinned host memory is copied directly.  Allocated on first use, freed with the
// context.
constexpr size_t kStagingBytes = size_t(16) << 20;
constexpr int kStagingSlots = 3;

struct HostStaging {
    void* buf[kStagingSlots] = {};
    cudaEvent_t ev[kStagingSlots] = {};  // the last device copy that used each buffer
    int next = 0;
    int threads = 1;
    bool ready = false;
    cudaError_t init() {
        if (ready) return cudaSuccess;
        for (int i = 0; i < kStagingSlots; ++i) {
            cudaError_t e = buf[i] ? cudaSuccess
                                   : cudaHostAlloc(&buf[i], kStagingBytes, cudaHostAllocPortable);
            if (e == cudaSuccess && !ev[i])
                e = cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming);
            if (e != cudaSuccess) return e;
        }
        // PSM_STAGING_THREADS host threads copy (default: half the processors, at most 8)
        int t = std::max(1, std::min(8, omp_get_num_procs() / 2));
        if (const char* v = std::getenv("PSM_STAGING_THREADS")) t = std::max(1, std::atoi(v));
        threads = t;
        ready = true;
        return cudaSuccess;
    }
    void release() {
        for (int i = 0; i < kStagingSlots; ++i) {
            if (ev[i]) cudaEventSynchronize(ev[i]);
            if (buf[i]) cudaFreeHost(buf[i]);
            if (ev[i]) cudaEventDestroy(ev[i]);
            buf[i] = nullptr;
            ev[i] = nullptr;
        }
        ready = false;
    }
};

}  // namespace

struct psm_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    Status st;
    bool have_geom = false, have_traces = false, have_vrms = false;
    // `data` holds the fp32 cube of the resident traces (false after a streamed forward,
    // whose kept inlines live in the staged storage only, and after least-squares migration)
    bool traces_readable = false;
    psm_geom g{};
    int ns = 0;
    int store = psm::kStoreF32;  // trace storage of the resident cube
    int variant = PSM_FWD_DEFAULT;
    std::vector<Job> jobs;       // one per distinct migrated inline
    std::vector<Job> jobs_all;   // one per output row (term counting)
    std::vector<std::pair<int, int>> copies;  // (dst row, src row) duplicated output rows
    // data: fp32 traces [n_il][n_xl][ns] as uploaded; pairs: the (d, d[t+1]-d) cube the
    // forward kernel stages
    DevBuf data, pairs, vrms, image, d_jobs, d_jobs_all, il_pos, t0, err, count;
    // 16-bit storage: words [n_il][n_xl][ns] (q[t] | q[t+1] << 16) and one scale per trace
    DevBuf words, scales;
    // adjoint: rows of each job (fold of duplicated output rows), image upload, job images
    std::vector<int> fold_map, fold_off;
    DevBuf d_fold_map, d_fold_off, img_in, fold;
    DevBuf d_copies;  // the repeated output rows as int2 (dst row, src row)
    // least-squares migration vectors: data space [n_tr][ns], image space [n_oi][n_ox][n_t]
    DevBuf cg_d, cg_r, cg_q, cg_m, cg_s, cg_p, cg_sc, cg_hist;
    // SEG-Y codec: the input trace records as uploaded, their cube positions, the output
    // records and their header sources / labels; a copy stream overlaps upload and decode
    DevBuf seg_rec, seg_pos, seg_out, seg_src, seg_il, seg_xl;
    int64_t seg_n = 0;
    int seg_rec_bytes = 0;
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t copied = nullptr;
    // psm_forward_host: the device-to-host stream, a second compute stream and the jobs in
    // wave order
    cudaStream_t d2h_stream = nullptr;
    cudaStream_t aux_stream = nullptr;
    DevBuf d_jobs_waves;
    // psm_forward_streamed: the next slab's new inlines staged during the current slab's
    // migration (fp32 rows of ns samples, Vrms rows), two slab images in turn, and the events
    // that order staging, placement and the image copies
    DevBuf str_tr, str_v, str_img[2];
    cudaEvent_t ev_placed = nullptr, ev_staged = nullptr, ev_done[2] = {nullptr, nullptr};
    // adjoint: 64-bit fixed-point window sums and an FP64 data cube (else fp32 atomics)
    bool adj_fixed = false;
    DevBuf adj64;
    // limit of the kernels' mbarrier waits (us; 0: the kernels' default of 4 s) and the
    // test-only failure injection (psm::kFault*), both read from the environment by psm_create
    unsigned wait_us = 0;
    int fault = 0;
    HostStaging staging;  // pageable host copies
};

namespace {

// Error-path knobs from the environment, for tests (read at each psm_create):
//   PSM_WAIT_LIMIT_MS   limit of every mbarrier wait in the kernels (default 4000 ms);
//   PSM_FAULT           "stall_producer": the forward producer leaves the first stage of
//                       each tile unfilled, so the consumers' wait runs out and the launch
//                       returns PSM_ERR_DEVICE; "nomem:K": the K-th device allocation from
//                       now on fails with PSM_ERR_NOMEM.
void read_fault_env(psm_ctx* c) {
    if (const char* w = std::getenv("PSM_WAIT_LIMIT_MS")) {
        const long long ms = std::atoll(w);
        if (ms > 0 && ms < 4000000) c->wait_us = static_cast<unsigned>(ms * 1000);
    }
    if (const char* a = std::getenv("PSM_ADJ_ACCUM"))  // "fixed": 64-bit fixed-point sums
        c->adj_fixed = std::strcmp(a, "fixed") == 0;
    if (const char* f = std::getenv("PSM_FAULT")) {
        if (!std::strcmp(f, "stall_producer")) c->fault = psm::kFaultStallProducer;
        if (!std::strncmp(f, "nomem:", 6)) g_fail_alloc.store(std::atoi(f + 6));
    }
}

// The repeated output rows of the ctx geometry, copied within image `img` in one launch.
cudaError_t copy_rows(psm_ctx* c, float* img, cudaStream_t s) {
    if (c->copies.empty()) return cudaSuccess;
    const size_t row = static_cast<size_t>(c->g.n_ox) * c->g.n_t;
    const size_t total = c->copies.size() * row;
    const unsigned blocks = static_cast<unsigned>(std::min<size_t>((total + 255) / 256, 148 * 16));
    psm::copy_rows_kernel<<<blocks, 256, 0, s>>>(img, c->d_copies.as<int2>(),
                                                  static_cast<int>(c->copies.size()), row);
    return cudaGetLastError();
}

FwdParams volume_params(psm_ctx* c) {
    FwdParams P{};
    P.pairs = c->pairs.as<float2>();
    P.words = c->words.as<uint32_t>();
    P.scales = c->scales.as<float>();
    P.vrms = c->vrms.as<float>();
    P.image = c->image.as<float>();
    P.jobs = c->d_jobs.as<Job>();
    P.il_pos = c->il_pos.as<int>();
    P.t0 = c->t0.as<float>();
    P.err = c->err.as<int>();
    P.wait_us = c->wait_us;
    P.fault = c->fault;
    P.compat_pad = c->g.compat_omp_pad != 0;
    P.n_ci = c->g.n_il;
    P.n_cx = c->g.n_xl;
    P.n_t = c->g.n_t;
    P.ns = c->ns;
    P.n_vx = c->g.n_xl;
    P.n_ox = c->g.n_ox;
    P.xoff = -c->g.pad_xl;
    P.max_inl = max_inline_window(c->jobs_all);
    P.stage_cap = stage_cap(c->ns, c->store);
    fill_consts(P, c->g.dt, c->g.d_il, c->g.d_xl, c->g.tan2_theta);
    return P;
}

// Host memory the CUDA driver copies through its own staging (not pinned or registered).
bool pageable(const void* p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();  // clear it: an unknown pointer is ordinary host memory
        return true;
    }
    return a.type == cudaMemoryTypeUnregistered;
}

// memcpy on `threads` host threads (one below 1 MiB).
void host_copy(void* dst, const void* src, size_t bytes, int threads) {
    if (threads <= 1 || bytes < (size_t(1) << 20)) {
        std::memcpy(dst, src, bytes);
        return;
    }
    const size_t per = ((bytes + threads - 1) / threads + 63) & ~size_t(63);
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int t = 0; t < threads; ++t) {
        const size_t o = std::min(bytes, per * t), e = std::min(bytes, o + per);
        if (e > o)
            std::memcpy(static_cast<char*>(dst) + o, static_cast<const char*>(src) + o, e - o);
    }
}

// `rows` rows of `width` bytes, consecutive in host memory, to the device at pitch dpitch,
// enqueued on s.  Returns once the host memory has been read (the device copies may still
// be running), as a copy from pageable memory does.
cudaError_t upload_rows(HostStaging& H, void* dst, size_t dpitch, const void* src, size_t width,
                        size_t rows, cudaStream_t s) {
    if (rows == 0 || width == 0) return cudaSuccess;
    if (!pageable(src) || width > kStagingBytes)
        return cudaMemcpy2DAsync(dst, dpitch, src, width, width, rows, cudaMemcpyHostToDevice, s);
    cudaError_t e = H.init();
    if (e != cudaSuccess) return e;
    const size_t per = kStagingBytes / width;  // rows per staging buffer
    for (size_t r = 0; r < rows; r += per) {
        const size_t n = std::min(per, rows - r);
        const int k = H.next;
        H.next = (k + 1) % kStagingSlots;
        if ((e = cudaEventSynchronize(H.ev[k])) != cudaSuccess) return e;  // buffer free
        host_copy(H.buf[k], static_cast<const char*>(src) + r * width, n * width, H.threads);
        if ((e = cudaMemcpy2DAsync(static_cast<char*>(dst) + r * dpitch, dpitch, H.buf[k], width,
                                   width, n, cudaMemcpyHostToDevice, s)) != cudaSuccess)
            return e;
        if ((e = cudaEventRecord(H.ev[k], s)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t upload(HostStaging& H, void* dst, const void* src, size_t bytes, cudaStream_t s) {
    if (bytes == 0) return cudaSuccess;
    if (!pageable(src)) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
    // whole staging buffers as rows, then the remainder
    const size_t full = bytes / kStagingBytes;
    cudaError_t e = upload_rows(H, dst, kStagingBytes, src, kStagingBytes, full, s);
    if (e != cudaSuccess || bytes == full * kStagingBytes) return e;
    const size_t o = full * kStagingBytes;
    return upload_rows(H, static_cast<char*>(dst) + o, bytes - o,
                       static_cast<const char*>(src) + o, bytes - o, 1, s);
}

// bytes of device memory to the host, after s's earlier work.  To pageable memory: through
// the staging buffers, returning once the host has every byte; to pinned memory: one copy
// enqueued on s.
cudaError_t download(HostStaging& H, void* dst, const void* src, size_t bytes, cudaStream_t s) {
    if (bytes == 0) return cudaSuccess;
    if (!pageable(dst)) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s);
    cudaError_t e = H.init();
    if (e != cudaSuccess) return e;
    const size_t n = (bytes + kStagingBytes - 1) / kStagingBytes;
    auto issue = [&](size_t i) -> cudaError_t {  // device copy of chunk i into buffer i % slots
        const int k = static_cast<int>(i % kStagingSlots);
        cudaError_t r = cudaEventSynchronize(H.ev[k]);  // the buffer's last use is over
        if (r != cudaSuccess) return r;
        const size_t o = i * kStagingBytes, len = std::min(kStagingBytes, bytes - o);
        r = cudaMemcpyAsync(H.buf[k], static_cast<const char*>(src) + o, len,
                            cudaMemcpyDeviceToHost, s);
        return r != cudaSuccess ? r : cudaEventRecord(H.ev[k], s);
    };
    for (size_t i = 0; i < std::min<size_t>(n, kStagingSlots); ++i)
        if ((e = issue(i)) != cudaSuccess) return e;
    for (size_t i = 0; i < n; ++i) {
        const int k = static_cast<int>(i % kStagingSlots);
        if ((e = cudaEventSynchronize(H.ev[k])) != cudaSuccess) return e;
        const size_t o = i * kStagingBytes, len = std::min(kStagingBytes, bytes - o);
        host_copy(static_cast<char*>(dst) + o, H.buf[k], len, H.threads);
        if (i + kStagingSlots < n && (e = issue(i + kStagingSlots)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

int read_device_error(psm_ctx* c) {
    int h = 0;
    PSM_CUDA_TRY(c->st, cudaMemcpyAsync(&h, c->err.p, sizeof(int), cudaMemcpyDeviceToHost,
                                        c->stream));
    PSM_CUDA_TRY(c->st, cudaStreamSynchronize(c->stream));
    if (h) return c->st.fail(PSM_ERR_DEVICE, "kernel reported device error flags " +
                                                 std::to_string(h));
    return PSM_OK;
}

}  // namespace

extern "C" {

const char* psm_version(void) { return "poststackmig3d-b200 0.1 (sm_100a)"; }

int psm_device_count(int* count) {
    if (!count) return PSM_ERR_ARG;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) n = 0;
    *count = n;
    return PSM_OK;
}

int psm_create(psm_ctx** out, int device) {
    if (!out) return PSM_ERR_ARG;
    *out = nullptr;
    psm_ctx* c = new (std::nothrow) psm_ctx();
    if (!c) return PSM_ERR_NOMEM;
    c->device = device;
    read_fault_env(c);
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return PSM_ERR_CUDA;
    }
    *out = c;
    return PSM_OK;
}

int psm_destroy(psm_ctx* c) {
    if (!c) return PSM_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    c->data.release();
    c->pairs.release();
    c->words.release();
    c->scales.release();
    c->vrms.release();
    c->image.release();
    c->d_jobs.release();
    c->d_jobs_all.release();
    c->il_pos.release();
    c->t0.release();
    c->err.release();
    c->count.release();
    for (DevBuf* b : {&c->d_fold_map, &c->d_fold_off, &c->img_in, &c->fold, &c->cg_d, &c->cg_r,
                      &c->cg_q, &c->cg_m, &c->cg_s, &c->cg_p, &c->cg_sc, &c->cg_hist,
                      &c->seg_rec, &c->seg_pos, &c->seg_out, &c->seg_src, &c->seg_il,
                      &c->seg_xl})
        b->release();
    if (c->copied) cudaEventDestroy(c->copied);
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    if (c->d2h_stream) cudaStreamDestroy(c->d2h_stream);
    if (c->aux_stream) cudaStreamDestroy(c->aux_stream);
    c->d_jobs_waves.release();
    c->d_copies.release();
    for (DevBuf* b : {&c->str_tr, &c->str_v, &c->str_img[0], &c->str_img[1], &c->adj64})
        b->release();
    for (cudaEvent_t e : {c->ev_placed, c->ev_staged, c->ev_done[0], c->ev_done[1]})
        if (e) cudaEventDestroy(e);
    c->staging.release();
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return PSM_OK;
}

const char* psm_last_error(const psm_ctx* c) { return c ? c->st.msg.c_str() : "null context"; }

int psm_stream(psm_ctx* c, void** s) {
    if (!c || !s) return PSM_ERR_ARG;
    *s = c->stream;
    return PSM_OK;
}

int psm_set_geometry(psm_ctx* c, const psm_geom* g, const int32_t* out_center) {
    if (!c || !g) return PSM_ERR_ARG;
    cudaSetDevice(c->device);
    std::string why;
    int rc = check_geometry(*g, &why);
    if (rc) return c->st.fail(rc, why);
    std::vector<Job> jobs, jobs_all;
    std::vector<std::pair<int, int>> copies;
    if (!plan_jobs(*g, out_center, jobs, jobs_all, copies))
        return c->st.fail(PSM_ERR_ARG, "out_center out of range");
    const int store = store_of(g->precision);
    const int ns = trace_stride(g->n_t);
    // nothing of the previous geometry stays usable, whether or not the allocations below
    // succeed
    c->have_geom = c->have_traces = c->have_vrms = c->traces_readable = false;
    c->g = *g;
    c->ns = ns;
    c->store = store;
    c->jobs.swap(jobs);
    c->jobs_all.swap(jobs_all);
    c->copies.swap(copies);
    const size_t n_tr = static_cast<size_t>(g->n_il) * g->n_xl;
    PSM_CUDA_TRY(c->st, c->data.ensure(n_tr * ns * sizeof(float)));
    PSM_CUDA_TRY(c->st, cudaMemsetAsync(c->data.p, 0, n_tr * ns * sizeof(float), c->stream));
    PSM_CUDA_TRY(c->st, c->pairs.ensure(n_tr * ns * sizeof(float2)));
    if (store != psm::kStoreF32) {
        PSM_CUDA_TRY(c->st, c->words.ensure(n_tr * ns * sizeof(uint32_t)));
        PSM_CUDA_TRY(c->st, c->scales.ensure(n_tr * sizeof(float)));
    }
    PSM_CUDA_TRY(c->st, c->vrms.ensure(n_tr * g->n_t * sizeof(float)));
    PSM_CUDA_TRY(c->st, c->image.ensure(static_cast<size_t>(g->n_oi) * g->n_ox * g->n_t *
                                        sizeof(float)));
    PSM_CUDA_TRY(c->st, c->d_jobs.ensure(c->jobs.size() * sizeof(Job)));
    PSM_CUDA_TRY(c->st, c->d_jobs_all.ensure(c->jobs_all.size() * sizeof(Job)));
    PSM_CUDA_TRY(c->st, c->il_pos.ensure(g->n_il * sizeof(int)));
    PSM_CUDA_TRY(c->st, c->t0.ensure(g->n_t * sizeof(float)));
    PSM_CUDA_TRY(c->st, c->err.ensure(sizeof(int)));
        std::vector<int> pos(g->n_il);
    for (int i = 0; i < g->n_il; ++i) pos[i] = i;
    std::vector<float> t0(g->n_t);
    for (int i = 0; i < g->n_t; ++i)
        t0[i] = static_cast<float>(static_cast<double>(i) * g->dt_seconds);  // main.cpp:216
    PSM_CUDA_TRY(c->st, cudaMemcpyAsync(c->d_jobs.p, c->jobs.data(), c->jobs.size() * sizeof(Job),
                                        cudaMemcpyHostToDevice, c->stream));
    PSM_CUDA_TRY(c->st, cudaMemcpyAsync(c->d_jobs_all.p, c->jobs_all.data(),
                                        c->jobs_all.size() * sizeof(Job),
                                        cudaMemcpyHostToDevice, c->stream));
    PSM_CUDA_TRY(c->st, cudaMemcpyAsync(c->il_pos.p, pos.data(), pos.size() * sizeof(int),
                                        cudaMemcpyHostToDevice, c->stream));
    PSM_CUDA_TRY(c->st, cudaMemcpyAsync(c->t0.p, t0.data(), t0.size() * sizeof(float),
                                        cudaMemcpyHostToDevice, c->stream));
    // adjoint: the output rows of every job (its own row, then the rows that repeat it)
    c->fold_map.clear();
    c->fold_off.assign(1, 0);
    for (const Job& j : c->jobs) {
        c->fold_map.push_back(j.row);
        for (const auto& cp : c->copies)
            if (cp.second == j.row) c->fold_map.push_back(cp.first);
        c->fold_off.push_back(static_cast<int>(c->fold_map.size()));
    }
    PSM_CUDA_TRY(c->st, c->d_fold_map.ensure(c->fold_map.size() * sizeof(int)));
    PSM_CUDA_TRY(c->st, c->d_fold_off.ensure(c->fold_off.size() * sizeof(int)));
    PSM_CUDA_TRY(c->st, cudaMemcpyAsync(c->d_fold_map.p, c->fold_map.data(),
                                        c->fold_map.size() * sizeof(int),
                                        cudaMemcpyHostToDevice, c->stream));
    PSM_CUDA_TRY(c->st, cudaMemcpyAsync(c->d_fold_off.p, c->fold_off.data(),
                                        c->fold_off.size() * sizeof(int),
                                        cudaMemcpyHostToDevice, c->stream));
    std::vector<int2> cps;
    for (const auto& cp : c->copies) cps.push_back(make_int2(cp.first, cp.second));
    PSM_CUDA_TRY(c->st, c->d_copies.ensure(std::max<size_t>(cps.size(), 1) * sizeof(int2)));
    if (!cps.empty())
        PSM_CUDA_TRY(c->st, cudaMemcpyAsync(c->d_copies.p, cps.data(), cps.size() * sizeof(int2),
                                            cudaMemcpyHostToDevice, c->stream));
    PSM_CUDA_TRY(c->st, cudaStreamSynchronize(c->stream));
    c->have_geom = true;
    c->have_traces = c->have_vrms = c->traces_readable = false;
    return PSM_OK;
}

int psm_set_traces(psm_ctx* c, const float* data) {
    if (!c || !data) return PSM_ERR_ARG;
    if (!c->have_geom) return c->st.fail(PSM_ERR_STATE, "psm_set_geometry first");
    cudaSetDevice(c->device);
    const size_t n_tr = static_cast<size_t>(c->g.n_il) * c->g.n_xl;
    PSM_CUDA_TRY(c->st, upload_rows(c->staging, c->data.p, c->ns * sizeof(float), data,
                                    c->g.n_t * sizeof(float), n_tr, c->stream));
    if (c->store == psm::kStoreF32)
        PSM_CUDA_TRY(c->st, build_pairs(c->data.as<float>(), c->pairs.as<float2>(), n_tr, c->ns,
                                        c->stream));
    else
        PSM_CUDA_TRY(c->st, quantize(c->data.as<float>(), c->words.as<uint32_t>(),
                                     c->scales.as<float>(), n_tr, c->ns, c->store, c->stream));
    PSM_CUDA_TRY(c->st, cudaStreamSynchronize(c->stream));
    c->have_traces = c->traces_readable = true;
    return PSM_OK;
}

int psm_get_traces(psm_ctx* c, float* data) {
    if (!c || !data) return PSM_ERR_ARG;
    if (!c->traces_readable) return c->st.fail(PSM_ERR_STATE, "no readable traces on the device");
    cudaSetDevice(c->device);
    const size_t n_tr = static_cast<size_t>(c->g.n_il) * c->g.n_xl;
    PSM_CUDA_TRY(c->st, cudaMemcpy2DAsync(data, c->g.n_t * sizeof(float), c->data.p,
                                          c->ns * sizeof(float), c->g.n_t * sizeof(float), n_tr,
                                          cudaMemcpyDeviceToHost, c->stream));
    PSM_CUDA_TRY(c->st, cudaStreamSynchronize(c->stream));
    return PSM_OK;
}

int psm_set_traces_segy(psm_ctx* c, const void* records, int64_t n_records, int32_t format,
                        const int32_t* position) {
    if (!c || n_records < 0 || (n_records && (!records || !position))) return PSM_ERR_ARG;
    if (!c->have_geom) return c->st.fail(PSM_ERR_STATE, "psm_set_geometry first");
    cudaSetDevice(c->device);
    const int64_t n_tr = static_cast<int64_t>(c->g.n_il) * c->g.n_xl;
    {  // every record fills at most one cube trace, every cube trace at most once
        std::vector<unsigned char> seen(static_cast<size_t>(n_tr), 0);
        for (int64_t r = 0; r < n_records; ++r) {
            const int32_t p = position[r];
            if (p < -1 || p >= n_tr || (p >= 0 && seen[p]++))
                return c->st.fail(PSM_ERR_ARG, "position " + std::to_string(r) +
                                                   ": out of range or repeated");
        }
    }
    const int rec_bytes = psm::kSegyTraceHeader + 4 * c->g.n_t;
    cudaStream_t s = c->stream;
    if (!c->copy_stream)
        PSM_CUDA_TRY(c->st, cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    if (!c->copied)
        PSM_CUDA_TRY(c->st, cudaEventCreateWithFlags(&c->copied, cudaEventDisableTiming));
    PSM_CUDA_TRY(c->st, c->seg_rec.ensure(static_cast<size_t>(n_records) * rec_bytes));
    PSM_CUDA_TRY(c->st, c->seg_pos.ensure(static_cast<size_t>(n_records) * sizeof(int32_t)));
    PSM_CUDA_TRY(c->st, cudaMemsetAsync(c->data.p, 0, n_tr * c->ns * sizeof(float), s));
    PSM_CUDA_TRY(c->st, cudaMemcpyAsync(c->seg_pos.p, position, n_records * sizeof(int32_t),
                                        cudaMemcpyHostToDevice, s));
    // chunks of about 32 MB: the copy of chunk k + 1 (copy stream) overlaps the decode of
    // chunk k (ctx stream) when the records are in pinned memory
    const int64_t per_chunk = std::max<int64_t>(1, (int64_t(32) << 20) / rec_bytes);
    PSM_CUDA_TRY(c->st, cudaEventRecord(c->copied, s));  // the copy stream follows the memsets
    PSM_CUDA_TRY(c->st, cudaStreamWaitEvent(c->copy_stream, c->copied, 0));
    for (int64_t r0 = 0; r0 < n_records; r0 += per_chunk) {
        const int64_t n = std::min(per_chunk, n_records - r0);
        PSM_CUDA_TRY(c->st, upload(c->staging, c->seg_rec.as<unsigned char>() + r0 * rec_bytes,
                                   static_cast<const unsigned char*>(records) + r0 * rec_bytes,
                                   static_cast<size_t>(n) * rec_bytes, c->copy_stream));
        PSM_CUDA_TRY(c->st, cudaEventRecord(c->copied, c->copy_stream));
        PSM_CUDA_TRY(c->st, cudaStreamWaitEvent(s, c->copied, 0));
        const unsigned blocks = static_cast<unsigned>(std::min<int64_t>((n + 7) / 8, 148 * 16));
        psm::segy_decode_kernel<<<blocks, 256, 0, s>>>(
            c->seg_rec.as<unsigned char>() + r0 * rec_bytes, n, rec_bytes, c->g.n_t, c->ns,
            format, c->seg_pos.as<int32_t>() + r0, c->data.as<float>());
        PSM_CUDA_TRY(c->st, cudaGetLastError());
    }
    if (c->store == psm::kStoreF32)
        PSM_CUDA_TRY(c->st, build_pairs(c->data.as<float>(), c->pairs.as<float2>(),
                                        static_cast<size_t>(n_tr), c->ns, s));
    else
        PSM_CUDA_TRY(c->st, quantize(c->data.as<float>(), c->words.as<uint32_t>(),
                                     c->scales.as<float>(), static_cast<size_t>(n_tr), c->ns,
                                     c->store, s));
    PSM_CUDA_TRY(c->st, cudaStreamSynchronize(s));
    c->seg_n = n_records;
    c->seg_rec_bytes = rec_bytes;
    c->have_traces = c->traces_readable = true;
    return PSM_OK;
}

int psm_set_image(psm_ctx* c, const float* image) {
    if (!c || !image) return PSM_ERR_ARG;
    if (!c->have_geom) return c->st.fail(PSM_ERR_STATE, "psm_set_geometry first");
    cudaSetDevice(c->device);
    const size_t n = static_cast<size_t>(c->g.n_oi) * c->g.n_ox * c->g.n_t;
    PSM_CUDA_TRY(c->st, cudaMemcpyAsync(c->image.p, image, n * sizeof(float),
                                        cudaMemcpyHostToDevice, c->stream));
    PSM_CUDA_TRY(c->st, cudaStreamSynchronize(c->stream));
    return PSM_OK;
}

int psm_get_image_segy(psm_ctx* c, void* out, int32_t format, const int32_t* source,
                       const int32_t* il_label, const int32_t* xl_label) {
    if (!c || !out || !source || !il_label || !xl_label) return PSM_ERR_ARG;
    if (!c->have_geom) return c->st.fail(PSM_ERR_STATE, "psm_set_geometry first");
    cudaSetDevice(c->device);
    const int64_t n_out = static_cast<int64_t>(c->g.n_oi) * c->g.n_ox;
    for (int64_t r = 0; r < n_out; ++r)
        if (source[r] < -1 || source[r] >= c->seg_n ||
            (source[r] >= 0 && c->seg_rec_bytes != psm::kSegyTraceHeader + 4 * c->g.n_t))
            return c->st.fail(PSM_ERR_ARG, "source " + std::to_string(r) +
                                               ": no such uploaded record");
    const int out_rec_bytes = psm::kSegyTraceHeader + 4 * c->g.n_t;
    cudaStream_t s = c->stream;
    PSM_CUDA_TRY(c->st, c->seg_out.ensure(static_cast<size_t>(n_out) * out_rec_bytes));
    PSM_CUDA_TRY(c->st, c->seg_src.ensure(static_cast<size_t>(n_out) * sizeof(int32_t)));
    PSM_CUDA_TRY(c->st, c->seg_il.ensure(c->g.n_oi * sizeof(int32_t)));
    PSM_CUDA_TRY(c->st, c->seg_xl.ensure(c->g.n_ox * sizeof(int32_t)));
    PSM_CUDA_TRY(c->st, cudaMemcpyAsync(c->seg_src.p, source, n_out * sizeof(int32_t),
                                        cudaMemcpyHostToDevice, s));
    PSM_CUDA_TRY(c->st, cudaMemcpyAsync(c->seg_il.p, il_label, c->g.n_oi * sizeof(int32_t),
                                        cudaMemcpyHostToDevice, s));
    PSM_CUDA_TRY(c->st, cudaMemcpyAsync(c->seg_xl.p, xl_label, c->g.n_ox * sizeof(int32_t),
                                        cudaMemcpyHostToDevice, s));
    const unsigned blocks = static_cast<unsigned>(std::min<int64_t>((n_out + 7) / 8, 148 * 16));
    psm::segy_encode_kernel<<<blocks, 256, 0, s>>>(
        c->image.as<float>(), n_out, c->g.n_ox, c->g.n_t, format, c->seg_src.as<int32_t>(),
        c->seg_rec.as<unsigned char>(), c->seg_rec_bytes, c->seg_il.as<int32_t>(),
        c->seg_xl.as<int32_t>(), c->seg_out.as<unsigned char>());
    PSM_CUDA_TRY(c->st, cudaGetLastError());
    PSM_CUDA_TRY(c->st, download(c->staging, out, c->seg_out.p,
                                 static_cast<size_t>(n_out) * out_rec_bytes, s));
    PSM_CUDA_TRY(c->st, cudaStreamSynchronize(s));
    return read_device_error(c);
}

int psm_get_vrms(psm_ctx* c, float* vrms) {
    if (!c || !vrms) return PSM_ERR_ARG;
    if (!c->have_vrms) return c->st.fail(PSM_ERR_STATE, "no Vrms set");
    cudaSetDevice(c->device);
    const size_t n = static_cast<size_t>(c->g.n_il) * c->g.n_xl * c->g.n_t;
    PSM_CUDA_TRY(c->st, download(c->staging, vrms, c->vrms.p, n * sizeof(float), c->stream));
    PSM_CUDA_TRY(c->st, cudaStreamSynchronize(c->stream));
    return PSM_OK;
}

}  // extern "C"

namespace {

// Upload n values to a temporary device buffer (freed by the caller's DevBuf).
template <class T>
cudaError_t upload(DevBuf& b, const T* host, size_t n, cudaStream_t s) {
    cudaError_t e = b.ensure(std::max<size_t>(n, 1) * sizeof(T));
    if (e != cudaSuccess || !n) return e;
    return cudaMemcpyAsync(b.p, host, n * sizeof(T), cudaMemcpyHostToDevice, s);
}

inline unsigned vrms_blocks(size_t n) {
    return static_cast<unsigned>(std::max<size_t>(1, std::min<size_t>((n + 255) / 256, 148 * 32)));
}

}  // namespace

extern "C" {

int psm_set_vrms_table(psm_ctx* c, const int32_t* p_il, const int32_t* p_xl,
                       const double* p_time, const float* p_v, int32_t n_points,
                       const int32_t* il_labels, const int32_t* xl_labels) {
    if (!c || n_points <= 0 || !p_il || !p_xl || !p_time || !p_v || !il_labels || !xl_labels)
        return PSM_ERR_ARG;
    if (!c->have_geom) return c->st.fail(PSM_ERR_STATE, "psm_set_geometry first");
    cudaSetDevice(c->device);
    float vmin = p_v[0];
    for (int32_t i = 1; i < n_points; ++i) vmin = std::min(vmin, p_v[i]);
    cudaStream_t s = c->stream;
    DevBuf d_il, d_xl, d_t, d_v, d_lil, d_lxl;
    PSM_CUDA_TRY(c->st, upload(d_il, p_il, n_points, s));
    PSM_CUDA_TRY(c->st, upload(d_xl, p_xl, n_points, s));
    PSM_CUDA_TRY(c->st, upload(d_t, p_time, n_points, s));
    PSM_CUDA_TRY(c->st, upload(d_v, p_v, n_points, s));
    PSM_CUDA_TRY(c->st, upload(d_lil, il_labels, c->g.n_il, s));
    PSM_CUDA_TRY(c->st, upload(d_lxl, xl_labels, c->g.n_xl, s));
    const size_t n = static_cast<size_t>(c->g.n_il) * c->g.n_xl * c->g.n_t;
    psm::vrms_table_kernel<<<vrms_blocks(n), 256, 0, s>>>(
        d_il.as<int32_t>(), d_xl.as<int32_t>(), d_t.as<double>(), d_v.as<float>(), n_points,
        vmin, d_lil.as<int32_t>(), d_lxl.as<int32_t>(), c->g.n_il, c->g.n_xl, c->g.n_t,
        c->g.dt_seconds, c->vrms.as<float>());
    PSM_CUDA_TRY(c->st, cudaGetLastError());
    PSM_CUDA_TRY(c->st, cudaStreamSynchronize(s));
    c->have_vrms = true;
    return PSM_OK;
}

int psm_set_vrms_grid(psm_ctx* c, const float* grid, const int32_t* g_il, int32_t g_nil,
                      const int32_t* g_xl, int32_t g_nxl, int32_t g_nt, double g_dt,
                      const int32_t* il_labels, const int32_t* xl_labels) {
    if (!c || !grid || !g_il || !g_xl || g_nil <= 0 || g_nxl <= 0 || g_nt <= 0 ||
        !(g_dt > 0.0) || !il_labels || !xl_labels)
        return PSM_ERR_ARG;
    if (!c->have_geom) return c->st.fail(PSM_ERR_STATE, "psm_set_geometry first");
    for (int32_t i = 1; i < g_nil; ++i)
        if (g_il[i] <= g_il[i - 1]) return c->st.fail(PSM_ERR_ARG, "grid inlines not increasing");
    for (int32_t i = 1; i < g_nxl; ++i)
        if (g_xl[i] <= g_xl[i - 1])
            return c->st.fail(PSM_ERR_ARG, "grid crosslines not increasing");
    cudaSetDevice(c->device);
    cudaStream_t s = c->stream;
    DevBuf d_grid, d_gil, d_gxl, d_lil, d_lxl;
    PSM_CUDA_TRY(c->st, upload(d_grid, grid, static_cast<size_t>(g_nil) * g_nxl * g_nt, s));
    PSM_CUDA_TRY(c->st, upload(d_gil, g_il, g_nil, s));
    PSM_CUDA_TRY(c->st, upload(d_gxl, g_xl, g_nxl, s));
    PSM_CUDA_TRY(c->st, upload(d_lil, il_labels, c->g.n_il, s));
    PSM_CUDA_TRY(c->st, upload(d_lxl, xl_labels, c->g.n_xl, s));
    const size_t n = static_cast<size_t>(c->g.n_il) * c->g.n_xl * c->g.n_t;
    psm::vrms_grid_kernel<<<vrms_blocks(n), 256, 0, s>>>(
        d_grid.as<float>(), d_gil.as<int32_t>(), g_nil, d_gxl.as<int32_t>(), g_nxl, g_nt, g_dt,
        d_lil.as<int32_t>(), d_lxl.as<int32_t>(), c->g.n_il, c->g.n_xl, c->g.n_t,
        c->g.dt_seconds, c->vrms.as<float>());
    PSM_CUDA_TRY(c->st, cudaGetLastError());
    PSM_CUDA_TRY(c->st, cudaStreamSynchronize(s));
    c->have_vrms = true;
    return PSM_OK;
}

int psm_set_vrms(psm_ctx* c, const float* vrms) {
    if (!c || !vrms) return PSM_ERR_ARG;
    if (!c->have_geom) return c->st.fail(PSM_ERR_STATE, "psm_set_geometry first");
    cudaSetDevice(c->device);
    const size_t n = static_cast<size_t>(c->g.n_il) * c->g.n_xl * c->g.n_t;
    PSM_CUDA_TRY(c->st, upload(c->staging, c->vrms.p, vrms, n * sizeof(float), c->stream));
    PSM_CUDA_TRY(c->st, cudaStreamSynchronize(c->stream));
    c->have_vrms = true;
    return PSM_OK;
}

int psm_forward_async(psm_ctx* c) {
    if (!c) return PSM_ERR_ARG;
    if (!c->have_geom || !c->have_traces || !c->have_vrms)
        return c->st.fail(PSM_ERR_STATE, "geometry, traces and vrms must be set");
    cudaSetDevice(c->device);
    PSM_CUDA_TRY(c->st, cudaMemsetAsync(c->err.p, 0, sizeof(int), c->stream));
    FwdParams P = volume_params(c);
    PSM_CUDA_TRY(c->st, launch_fwd(P, static_cast<int>(c->jobs.size()),
                                   c->g.amp_correction != 0, c->variant, c->stream, c->store,
                                   c->g.compensated != 0));
    // padded output inlines repeat the migrated edge inline (main.cpp:268-285)
    PSM_CUDA_TRY(c->st, copy_rows(c, c->image.as<float>(), c->stream));
    return PSM_OK;
}

int psm_set_variant(psm_ctx* c, int variant) {
    if (!c || variant < 0 || variant >= PSM_FWD_N_VARIANTS) return PSM_ERR_ARG;
    c->variant = variant;
    return PSM_OK;
}

int psm_get_variant(psm_ctx* c, int* variant) {
    if (!c || !variant) return PSM_ERR_ARG;
    *variant = effective_variant(c->variant, c->store, c->g.compensated != 0);
    return PSM_OK;
}

int psm_autotune(psm_ctx* c, float* ms, int* best) {
    if (!c) return PSM_ERR_ARG;
    if (!c->have_geom || !c->have_traces || !c->have_vrms)
        return c->st.fail(PSM_ERR_STATE, "geometry, traces and vrms must be set");
    cudaSetDevice(c->device);
    cudaEvent_t e0, e1;
    PSM_CUDA_TRY(c->st, cudaEventCreate(&e0));
    PSM_CUDA_TRY(c->st, cudaEventCreate(&e1));
    int pick = kDefaultVariant;
    float pick_ms = 3.0e38f;
    int rc = PSM_OK;
    for (int v = 1; v < PSM_FWD_N_VARIANTS && rc == PSM_OK; ++v) {
        if (effective_variant(v, c->store, c->g.compensated != 0) != v) continue;  // same kernel
        c->variant = v;
        float t = 0.0f;
        if ((rc = psm_forward_async(c)) != PSM_OK) break;  // warm (first launch, attribute)
        cudaEventRecord(e0, c->stream);
        if ((rc = psm_forward_async(c)) != PSM_OK) break;
        cudaEventRecord(e1, c->stream);
        if ((rc = psm_synchronize(c)) != PSM_OK) break;
        cudaEventElapsedTime(&t, e0, e1);
        if (ms) ms[v] = t;
        if (t < pick_ms) {
            pick_ms = t;
            pick = v;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->variant = pick;
    if (rc == PSM_OK && best) *best = pick;
    return rc;
}

int psm_synchronize(psm_ctx* c) {
    if (!c) return PSM_ERR_ARG;
    cudaSetDevice(c->device);
    PSM_CUDA_TRY(c->st, cudaStreamSynchronize(c->stream));
    return read_device_error(c);
}

int psm_image_device(psm_ctx* c, float** dev_image) {
    if (!c || !dev_image) return PSM_ERR_ARG;
    if (!c->have_geom) return c->st.fail(PSM_ERR_STATE, "psm_set_geometry first");
    *dev_image = c->image.as<float>();
    return PSM_OK;
}

int psm_get_image(psm_ctx* c, float* image) {
    if (!c || !image) return PSM_ERR_ARG;
    if (!c->have_geom) return c->st.fail(PSM_ERR_STATE, "psm_set_geometry first");
    cudaSetDevice(c->device);
    const size_t n = static_cast<size_t>(c->g.n_oi) * c->g.n_ox * c->g.n_t;
    PSM_CUDA_TRY(c->st, download(c->staging, image, c->image.p, n * sizeof(float), c->stream));
    PSM_CUDA_TRY(c->st, cudaStreamSynchronize(c->stream));
    return read_device_error(c);
}

int psm_forward(psm_ctx* c, float* image) {
    if (!c || !image) return PSM_ERR_ARG;
    int r = psm_forward_async(c);
    if (r) return r;
    return psm_get_image(c, image);
}

}  // extern "C"

namespace {

// psm_forward_host's pipeline.  after_launches (may be empty) runs once every upload and
// launch is enqueued, while the last waves migrate (psm_forward_streamed stages the next
// slab's inlines there).
int forward_waves(psm_ctx* c, const float* traces, const float* vrms, float* image,
                  const std::function<int()>& after_launches) {
    const psm_geom& g = c->g;
    cudaStream_t s = c->stream;
    for (cudaStream_t* t : {&c->copy_stream, &c->d2h_stream, &c->aux_stream})
        if (!*t) PSM_CUDA_TRY(c->st, cudaStreamCreateWithFlags(t, cudaStreamNonBlocking));
    // Inputs go up in blocks of consecutive inlines: trace block b (then its pair cube or 16-bit
    // words, built on the copy stream), and Vrms block v once the trace blocks that the output
    // inlines of block v read are up (an output inline needs its whole buffer, which reaches
    // about m_il + pad_il inlines ahead, but only its own Vrms row).  A job runs in the wave of
    // the first upload after which its buffer and Vrms row are resident.  Waves alternate
    // between two compute streams, so that one launch's tail of finishing CTAs overlaps the
    // next launch instead of idling SMs; the last wave is cut in two so that most of its rows
    // stream back while the rest migrate.  Each wave is enqueued right after the upload that
    // completes its inputs: a copy from pageable memory returns only once the host has staged
    // it, and the waves already enqueued migrate meanwhile.  The image rows' copies to the host
    // are enqueued after every upload and launch: into pageable memory such a copy returns only
    // once it is done, which would hold the next upload back until the wave has finished.
    const int n_blocks = std::min(g.n_il, 16);
    auto block_end = [&](int b) { return static_cast<int>(int64_t(b + 1) * g.n_il / n_blocks); };
    auto block_of = [&](int inl) {  // block holding inline inl
        int b = 0;
        while (block_end(b) <= inl) ++b;
        return b;
    };
    const int n_jobs = static_cast<int>(c->jobs.size());
    // Vrms block v goes up after trace block lead[v]: the last trace block any job of v reads
    std::vector<int> lead(n_blocks, 0);
    for (int k = 0; k < n_jobs; ++k) {
        const Job& j = c->jobs[k];
        const int v = block_of(j.vrow);
        lead[v] = std::max(lead[v], block_of(std::max(j.i1, 1) - 1));
    }
    for (int v = 1; v < n_blocks; ++v) lead[v] = std::max(lead[v], lead[v - 1]);
    std::vector<std::pair<int, int>> units;  // upload order: (0 traces / 1 Vrms, block)
    std::vector<int> t_unit(n_blocks), v_unit(n_blocks);
    for (int b = 0, v = 0; b < n_blocks; ++b) {
        t_unit[b] = static_cast<int>(units.size());
        units.emplace_back(0, b);
        for (; v < n_blocks && lead[v] <= b; ++v) {
            v_unit[v] = static_cast<int>(units.size());
            units.emplace_back(1, v);
        }
    }
    const int n_units = static_cast<int>(units.size());
    std::vector<std::vector<int>> wave(n_units);
    for (int k = 0; k < n_jobs; ++k) {
        const Job& j = c->jobs[k];
        const int u = std::max(t_unit[block_of(std::max(j.i1, 1) - 1)], v_unit[block_of(j.vrow)]);
        wave[u].push_back(k);
    }
    int last = n_units - 1;
    while (last > 0 && wave[last].empty()) --last;
    std::vector<Job> order;
    std::vector<std::pair<int, int>> chunks;  // (first job in order, count)
    std::vector<int> chunk_unit;              // upload the chunk waits for
    for (int u = 0; u < n_units; ++u) {
        const size_t w = wave[u].size();
        const size_t chunk_jobs = u == last && w >= 16 ? (w * 3 + 3) / 4 : std::max<size_t>(w, 1);
        for (size_t i = 0; i < w; i += chunk_jobs) {
            const int n = static_cast<int>(std::min<size_t>(chunk_jobs, w - i));
            chunks.emplace_back(static_cast<int>(order.size()), n);
            chunk_unit.push_back(u);
            for (int t = 0; t < n; ++t) order.push_back(c->jobs[wave[u][i + t]]);
        }
    }
    // rows each job's image fills: its own, then the rows that repeat it
    std::vector<std::vector<int>> dup(static_cast<size_t>(g.n_oi));
    for (const auto& cp : c->copies) dup[cp.second].push_back(cp.first);
    PSM_CUDA_TRY(c->st, c->d_jobs_waves.ensure(std::max<size_t>(order.size(), 1) * sizeof(Job)));
    PSM_CUDA_TRY(c->st, cudaMemcpyAsync(c->d_jobs_waves.p, order.data(), order.size() * sizeof(Job),
                                        cudaMemcpyHostToDevice, s));
    PSM_CUDA_TRY(c->st, cudaMemsetAsync(c->err.p, 0, sizeof(int), s));
    // events: one per upload, one per chunk, the start and the second stream's end
    std::vector<cudaEvent_t> ev(n_units + chunks.size() + 2, nullptr);
    for (auto& e : ev) {
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
            for (auto& d : ev)
                if (d) cudaEventDestroy(d);
            return c->st.fail(PSM_ERR_CUDA, "cudaEventCreateWithFlags failed");
        }
    }
    struct EventGuard {
        std::vector<cudaEvent_t>& e;
        ~EventGuard() {
            for (auto& d : e) cudaEventDestroy(d);
        }
    } guard{ev};
    cudaEvent_t ev_start = ev[n_units + chunks.size()], ev_aux = ev[n_units + chunks.size() + 1];
    // the copy and second compute streams start after the ctx stream's earlier work (jobs,
    // error word)
    PSM_CUDA_TRY(c->st, cudaEventRecord(ev_start, s));
    PSM_CUDA_TRY(c->st, cudaStreamWaitEvent(c->copy_stream, ev_start, 0));
    PSM_CUDA_TRY(c->st, cudaStreamWaitEvent(c->aux_stream, ev_start, 0));
    const size_t per_il = static_cast<size_t>(g.n_xl) * g.n_t;
    const size_t row = static_cast<size_t>(g.n_ox) * g.n_t;
    FwdParams P = volume_params(c);
    bool aux_used = false;
    size_t k = 0;  // next chunk
    struct RowCopy {
        size_t chunk, first, count;  // image rows [first, first + count) of chunk
    };
    std::vector<RowCopy> row_copies;
    for (int u = 0; u < n_units; ++u) {
        const int b = units[u].second;
        const int lo = b ? block_end(b - 1) : 0, hi = block_end(b);
        const size_t r0 = size_t(lo) * g.n_xl, rows = size_t(hi - lo) * g.n_xl;
        cudaStream_t cs = c->copy_stream;
        if (units[u].first == 0) {
            PSM_CUDA_TRY(c->st, upload_rows(c->staging, c->data.as<float>() + r0 * c->ns,
                                            c->ns * sizeof(float), traces + lo * per_il,
                                            g.n_t * sizeof(float), rows, cs));
            if (c->store == psm::kStoreF32)
                PSM_CUDA_TRY(c->st, build_pairs(c->data.as<float>() + r0 * c->ns,
                                                c->pairs.as<float2>() + r0 * c->ns, rows, c->ns,
                                                cs));
            else
                PSM_CUDA_TRY(c->st, quantize(c->data.as<float>() + r0 * c->ns,
                                             c->words.as<uint32_t>() + r0 * c->ns,
                                             c->scales.as<float>() + r0, rows, c->ns, c->store,
                                             cs));
        } else {
            PSM_CUDA_TRY(c->st, upload(c->staging, c->vrms.as<float>() + lo * per_il,
                                       vrms + lo * per_il, rows * g.n_t * sizeof(float), cs));
        }
        PSM_CUDA_TRY(c->st, cudaEventRecord(ev[u], cs));
        for (; k < chunks.size() && chunk_unit[k] == u; ++k) {  // the waves this upload frees
            cudaStream_t ks = (k % 2 == 0) ? s : c->aux_stream;
            aux_used = aux_used || ks != s;
            PSM_CUDA_TRY(c->st, cudaStreamWaitEvent(ks, ev[u], 0));
            FwdParams Q = P;
            Q.jobs = c->d_jobs_waves.as<Job>() + chunks[k].first;
            PSM_CUDA_TRY(c->st, launch_fwd(Q, chunks[k].second, g.amp_correction != 0,
                                           c->variant, ks, c->store, g.compensated != 0));
            std::vector<int> out_rows;
            for (int t = 0; t < chunks[k].second; ++t) {
                const int r = order[chunks[k].first + t].row;
                out_rows.push_back(r);
                for (int d : dup[r]) {  // padded output inlines repeat the edge inline
                    PSM_CUDA_TRY(c->st, cudaMemcpyAsync(c->image.as<float>() + d * row,
                                                        c->image.as<float>() + r * row,
                                                        row * sizeof(float),
                                                        cudaMemcpyDeviceToDevice, ks));
                    out_rows.push_back(d);
                }
            }
            PSM_CUDA_TRY(c->st, cudaEventRecord(ev[n_units + k], ks));
            std::sort(out_rows.begin(), out_rows.end());
            for (size_t i = 0; i < out_rows.size();) {  // runs of consecutive rows
                size_t e = i + 1;
                while (e < out_rows.size() && out_rows[e] == out_rows[e - 1] + 1) ++e;
                row_copies.push_back({k, static_cast<size_t>(out_rows[i]), e - i});
                i = e;
            }
        }
    }
    if (after_launches) {
        const int r = after_launches();
        if (r) return r;
    }
    for (size_t i = 0; i < row_copies.size(); ++i) {
        const RowCopy& rc = row_copies[i];
        if (i == 0 || row_copies[i - 1].chunk != rc.chunk)
            PSM_CUDA_TRY(c->st, cudaStreamWaitEvent(c->d2h_stream, ev[n_units + rc.chunk], 0));
        PSM_CUDA_TRY(c->st, download(c->staging, image + rc.first * row,
                                     c->image.as<float>() + rc.first * row,
                                     rc.count * row * sizeof(float), c->d2h_stream));
    }
    // the ctx stream's later work follows both compute streams and the uploads
    PSM_CUDA_TRY(c->st, cudaEventRecord(ev_aux, aux_used ? c->aux_stream : c->copy_stream));
    PSM_CUDA_TRY(c->st, cudaStreamWaitEvent(s, ev_aux, 0));
    if (aux_used) {
        PSM_CUDA_TRY(c->st, cudaEventRecord(ev_start, c->copy_stream));
        PSM_CUDA_TRY(c->st, cudaStreamWaitEvent(s, ev_start, 0));
    }
    PSM_CUDA_TRY(c->st, cudaStreamSynchronize(c->d2h_stream));
    PSM_CUDA_TRY(c->st, cudaStreamSynchronize(s));
    c->have_traces = c->have_vrms = c->traces_readable = true;
    return read_device_error(c);
}

}  // namespace

extern "C" {

int psm_forward_host(psm_ctx* c, const float* traces, const float* vrms, float* image) {
    if (!c || !traces || !vrms || !image) return PSM_ERR_ARG;
    if (!c->have_geom) return c->st.fail(PSM_ERR_STATE, "psm_set_geometry first");
    cudaSetDevice(c->device);
    return forward_waves(c, traces, vrms, image, {});
}

}  // extern "C"

// ---------------------------------------------------------------------------- adjoint, LSM

namespace {

// Samples per adjoint ring stage: 48 KB stages (32 KB for 3 CTAs per SM) of 4-byte fp32 sums
// or 8-byte fixed-point sums, and at least one whole trace.
inline int adj_stage_cap(int ns, int minb, int eb) {
    return std::max((minb == 4 ? 20480 : minb == 3 ? 32768 : 49152) / eb, ns);
}

template <bool AMP, int MINB, bool FIX>
cudaError_t launch_adj(const psm::AdjParams& A, dim3 grid, dim3 block, size_t smem,
                       cudaStream_t s) {
    cudaError_t e = cudaFuncSetAttribute(psm::adj_kernel<AMP, MINB, FIX>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    psm::adj_kernel<AMP, MINB, FIX><<<grid, block, smem, s>>>(A);
    return cudaGetLastError();
}

inline unsigned grid_for(size_t n) {
    return static_cast<unsigned>(std::max<size_t>(1, std::min<size_t>((n + 255) / 256, 148 * 8)));
}

// M^T: image rows [n_oi][n_ox][n_t] (device) -> data [n_il*n_xl][ns] (device, overwritten).
int adjoint_dev(psm_ctx* c, const float* d_rows, float* d_out) {
    const size_t row = static_cast<size_t>(c->g.n_ox) * c->g.n_t;
    const size_t n_tr = static_cast<size_t>(c->g.n_il) * c->g.n_xl;
    const int n_jobs = static_cast<int>(c->jobs.size());
    const float* job_img = d_rows;  // without repeated rows, job k is output row k
    if (!c->copies.empty()) {
        PSM_CUDA_TRY(c->st, c->fold.ensure(static_cast<size_t>(n_jobs) * row * sizeof(float)));
        psm::fold_rows_kernel<<<grid_for(n_jobs * row), 256, 0, c->stream>>>(
            d_rows, c->d_fold_map.as<int>(), c->d_fold_off.as<int>(), n_jobs, row,
            c->fold.as<float>());
        PSM_CUDA_TRY(c->st, cudaGetLastError());
        job_img = c->fold.as<float>();
    }
    const bool fix = c->adj_fixed;
    const size_t n_data = n_tr * c->ns;
    psm::AdjParams A{};
    A.F = volume_params(c);
    A.image = job_img;
    A.data = d_out;
    if (fix) {  // FP64 data cube, converted to d_out afterwards
        PSM_CUDA_TRY(c->st, c->adj64.ensure(n_data * sizeof(double)));
        PSM_CUDA_TRY(c->st, cudaMemsetAsync(c->adj64.p, 0, n_data * sizeof(double), c->stream));
        A.data64 = c->adj64.as<double>();
    } else {
        PSM_CUDA_TRY(c->st, cudaMemsetAsync(d_out, 0, n_data * sizeof(float), c->stream));
    }
    const int eb = fix ? 8 : 4;
    // 4 CTAs per SM (fp32 sums) when their 20 KB stages and the inline tables fit a quarter
    // of the SM, else 3 with 32 KB stages, else 2
    A.F.stage_cap = adj_stage_cap(c->ns, 4, eb);
    size_t smem = psm::adj_layout(A.F.max_inl, A.F.stage_cap, eb).total;
    const bool o4 = !fix && smem <= 56 * 1024;
    bool o3 = false;
    if (!o4) {
        A.F.stage_cap = adj_stage_cap(c->ns, 3, eb);
        smem = psm::adj_layout(A.F.max_inl, A.F.stage_cap, eb).total;
        o3 = smem <= 75 * 1024;
    }
    if (!o4 && !o3) {
        A.F.stage_cap = adj_stage_cap(c->ns, 2, eb);
        smem = psm::adj_layout(A.F.max_inl, A.F.stage_cap, eb).total;
    }
    if (smem > kMaxDynSmem)
        return c->st.fail(PSM_ERR_UNSUPPORTED, "n_t / aperture too large for the adjoint ring");
    if (n_jobs > 65535) return c->st.fail(PSM_ERR_UNSUPPORTED, "more than 65535 output inlines");
    dim3 grid((c->g.n_ox + psm::kTX - 1) / psm::kTX, n_jobs,
              (c->g.n_t + psm::kTT - 1) / psm::kTT);
    dim3 block(32 * (psm::kTX + 1));
    const bool amp = c->g.amp_correction != 0;
    cudaError_t e;
    if (fix)
        e = o3 ? (amp ? launch_adj<true, 3, true>(A, grid, block, smem, c->stream)
                      : launch_adj<false, 3, true>(A, grid, block, smem, c->stream))
               : (amp ? launch_adj<true, 2, true>(A, grid, block, smem, c->stream)
                      : launch_adj<false, 2, true>(A, grid, block, smem, c->stream));
    else if (o4)
        e = amp ? launch_adj<true, 4, false>(A, grid, block, smem, c->stream)
                : launch_adj<false, 4, false>(A, grid, block, smem, c->stream);
    else
        e = o3 ? (amp ? launch_adj<true, 3, false>(A, grid, block, smem, c->stream)
                      : launch_adj<false, 3, false>(A, grid, block, smem, c->stream))
               : (amp ? launch_adj<true, 2, false>(A, grid, block, smem, c->stream)
                      : launch_adj<false, 2, false>(A, grid, block, smem, c->stream));
    PSM_CUDA_TRY(c->st, e);
    if (fix) {
        psm::f64_to_f32_kernel<<<grid_for(n_data), 256, 0, c->stream>>>(c->adj64.as<double>(),
                                                                         d_out, n_data);
        PSM_CUDA_TRY(c->st, cudaGetLastError());
    }
    return PSM_OK;
}

// M: data [n_il*n_xl][ns] (device, zero tail) -> image rows (device).  Rebuilds the pair
// cube from d_vec.
int forward_dev(psm_ctx* c, const float* d_vec, float* d_img) {
    const size_t n_tr = static_cast<size_t>(c->g.n_il) * c->g.n_xl;
    PSM_CUDA_TRY(c->st, build_pairs(d_vec, c->pairs.as<float2>(), n_tr, c->ns, c->stream));
    FwdParams P = volume_params(c);
    P.image = d_img;
    P.stage_cap = stage_cap(c->ns);  // the operator pair of CG is the fp32 one
    PSM_CUDA_TRY(c->st, launch_fwd(P, static_cast<int>(c->jobs.size()),
                                   c->g.amp_correction != 0, c->variant, c->stream,
                                   psm::kStoreF32, c->g.compensated != 0));
    PSM_CUDA_TRY(c->st, copy_rows(c, d_img, c->stream));
    return PSM_OK;
}

int dot_dev(psm_ctx* c, const float* a, const float* b, size_t n, double* out) {
    PSM_CUDA_TRY(c->st, cudaMemsetAsync(out, 0, sizeof(double), c->stream));
    psm::dot_kernel<<<grid_for(n), 256, 0, c->stream>>>(a, b, n, out);
    PSM_CUDA_TRY(c->st, cudaGetLastError());
    return PSM_OK;
}

}  // namespace

extern "C" {

int psm_adjoint(psm_ctx* c, const float* image, float* data) {
    if (!c || !image || !data) return PSM_ERR_ARG;
    if (!c->have_geom || !c->have_vrms)
        return c->st.fail(PSM_ERR_STATE, "geometry and vrms must be set");
    cudaSetDevice(c->device);
    const size_t n_img = static_cast<size_t>(c->g.n_oi) * c->g.n_ox * c->g.n_t;
    const size_t n_tr = static_cast<size_t>(c->g.n_il) * c->g.n_xl;
    PSM_CUDA_TRY(c->st, c->img_in.ensure(n_img * sizeof(float)));
    PSM_CUDA_TRY(c->st, c->cg_q.ensure(n_tr * c->ns * sizeof(float)));
    PSM_CUDA_TRY(c->st, cudaMemsetAsync(c->err.p, 0, sizeof(int), c->stream));
    PSM_CUDA_TRY(c->st, upload(c->staging, c->img_in.p, image, n_img * sizeof(float), c->stream));
    int r = adjoint_dev(c, c->img_in.as<float>(), c->cg_q.as<float>());
    if (r) return r;
    PSM_CUDA_TRY(c->st, cudaMemcpy2DAsync(data, c->g.n_t * sizeof(float), c->cg_q.p,
                                          c->ns * sizeof(float), c->g.n_t * sizeof(float), n_tr,
                                          cudaMemcpyDeviceToHost, c->stream));
    PSM_CUDA_TRY(c->st, cudaStreamSynchronize(c->stream));
    return read_device_error(c);
}

int psm_adjoint_async(psm_ctx* c) {
    if (!c) return PSM_ERR_ARG;
    if (!c->have_geom || !c->have_vrms)
        return c->st.fail(PSM_ERR_STATE, "geometry and vrms must be set");
    cudaSetDevice(c->device);
    PSM_CUDA_TRY(c->st, cudaMemsetAsync(c->err.p, 0, sizeof(int), c->stream));
    int r = adjoint_dev(c, c->image.as<float>(), c->data.as<float>());
    if (r) return r;
    c->have_traces = false;      // the staged storage still holds the earlier traces
    c->traces_readable = true;   // the fp32 cube holds M^T image
    return PSM_OK;
}

int psm_forward_device(psm_ctx* c, const float* d_data, float* d_image) {
    if (!c || !d_data || !d_image) return PSM_ERR_ARG;
    if (!c->have_geom || !c->have_vrms)
        return c->st.fail(PSM_ERR_STATE, "geometry and vrms must be set");
    if (c->store != psm::kStoreF32 || c->g.compensated)
        return c->st.fail(PSM_ERR_UNSUPPORTED, "device operators take fp32 storage only");
    cudaSetDevice(c->device);
    const size_t n_tr = static_cast<size_t>(c->g.n_il) * c->g.n_xl;
    PSM_CUDA_TRY(c->st, cudaMemsetAsync(c->err.p, 0, sizeof(int), c->stream));
    // rows of n_t samples into the fp32 cube's rows of ns (their tails stay zero)
    PSM_CUDA_TRY(c->st, cudaMemcpy2DAsync(c->data.p, c->ns * sizeof(float), d_data,
                                          c->g.n_t * sizeof(float), c->g.n_t * sizeof(float),
                                          n_tr, cudaMemcpyDeviceToDevice, c->stream));
    const int r = forward_dev(c, c->data.as<float>(), d_image);
    if (r) return r;
    c->have_traces = c->traces_readable = true;
    return PSM_OK;
}

int psm_adjoint_device(psm_ctx* c, const float* d_image, float* d_data) {
    if (!c || !d_image || !d_data) return PSM_ERR_ARG;
    if (!c->have_geom || !c->have_vrms)
        return c->st.fail(PSM_ERR_STATE, "geometry and vrms must be set");
    cudaSetDevice(c->device);
    const size_t n_tr = static_cast<size_t>(c->g.n_il) * c->g.n_xl;
    PSM_CUDA_TRY(c->st, c->cg_q.ensure(n_tr * c->ns * sizeof(float)));
    PSM_CUDA_TRY(c->st, cudaMemsetAsync(c->err.p, 0, sizeof(int), c->stream));
    const int r = adjoint_dev(c, d_image, c->cg_q.as<float>());
    if (r) return r;
    PSM_CUDA_TRY(c->st, cudaMemcpy2DAsync(d_data, c->g.n_t * sizeof(float), c->cg_q.p,
                                          c->ns * sizeof(float), c->g.n_t * sizeof(float), n_tr,
                                          cudaMemcpyDeviceToDevice, c->stream));
    return PSM_OK;
}

int psm_lsm_cg(psm_ctx* c, const float* data, float* image, int iters, double* resid) {
    if (!c || !data || !image || iters < 0) return PSM_ERR_ARG;
    if (!c->have_geom || !c->have_vrms)
        return c->st.fail(PSM_ERR_STATE, "geometry and vrms must be set");
    cudaSetDevice(c->device);
    const size_t n_tr = static_cast<size_t>(c->g.n_il) * c->g.n_xl;
    const size_t nd = n_tr * c->ns;
    const size_t nm = static_cast<size_t>(c->g.n_oi) * c->g.n_ox * c->g.n_t;
    cudaStream_t s = c->stream;
    for (DevBuf* b : {&c->cg_d, &c->cg_r, &c->cg_q})
        PSM_CUDA_TRY(c->st, b->ensure(nd * sizeof(float)));
    for (DevBuf* b : {&c->cg_m, &c->cg_s, &c->cg_p})
        PSM_CUDA_TRY(c->st, b->ensure(nm * sizeof(float)));
    PSM_CUDA_TRY(c->st, c->cg_sc.ensure(8 * sizeof(double)));
    PSM_CUDA_TRY(c->st, c->cg_hist.ensure((iters + 1) * sizeof(double)));
    float *d = c->cg_d.as<float>(), *r = c->cg_r.as<float>(), *q = c->cg_q.as<float>();
    float *m = c->cg_m.as<float>(), *sv = c->cg_s.as<float>(), *p = c->cg_p.as<float>();
    double *sc = c->cg_sc.as<double>(), *hist = c->cg_hist.as<double>();
    PSM_CUDA_TRY(c->st, cudaMemsetAsync(c->err.p, 0, sizeof(int), s));
    PSM_CUDA_TRY(c->st, cudaMemsetAsync(d, 0, nd * sizeof(float), s));
    PSM_CUDA_TRY(c->st, upload_rows(c->staging, d, c->ns * sizeof(float), data,
                                    c->g.n_t * sizeof(float), n_tr, s));
    PSM_CUDA_TRY(c->st, cudaMemcpyAsync(r, d, nd * sizeof(float), cudaMemcpyDeviceToDevice, s));
    PSM_CUDA_TRY(c->st, cudaMemsetAsync(m, 0, nm * sizeof(float), s));
    PSM_CUDA_TRY(c->st, cudaMemsetAsync(sc, 0, 8 * sizeof(double), s));
    int rc;
    // CGLS: r = d - M^T m, s = M r, p = s, gamma = <s, s>
    if ((rc = dot_dev(c, r, r, nd, hist))) return rc;
    if ((rc = forward_dev(c, r, sv))) return rc;
    PSM_CUDA_TRY(c->st, cudaMemcpyAsync(p, sv, nm * sizeof(float), cudaMemcpyDeviceToDevice, s));
    if ((rc = dot_dev(c, sv, sv, nm, sc + 0))) return rc;
    for (int k = 0; k < iters; ++k) {
        if ((rc = adjoint_dev(c, p, q))) return rc;                   // q = M^T p
        if ((rc = dot_dev(c, q, q, nd, sc + 1))) return rc;           // delta
        psm::cg_alpha_kernel<<<1, 1, 0, s>>>(sc);                     // alpha = gamma / delta
        psm::cg_update_kernel<<<grid_for(nm + nd), 256, 0, s>>>(m, p, nm, r, q, nd, sc);
        if ((rc = dot_dev(c, r, r, nd, hist + k + 1))) return rc;     // ||r||^2
        if ((rc = forward_dev(c, r, sv))) return rc;                  // s = M r
        if ((rc = dot_dev(c, sv, sv, nm, sc + 2))) return rc;         // gamma_new
        psm::cg_beta_kernel<<<1, 1, 0, s>>>(sc);                      // beta, gamma
        psm::cg_direction_kernel<<<grid_for(nm), 256, 0, s>>>(p, sv, nm, sc);  // p = s + beta p
        PSM_CUDA_TRY(c->st, cudaGetLastError());
    }
    PSM_CUDA_TRY(c->st, download(c->staging, image, m, nm * sizeof(float), s));
    std::vector<double> h(iters + 1);
    PSM_CUDA_TRY(c->st, cudaMemcpyAsync(h.data(), hist, (iters + 1) * sizeof(double),
                                        cudaMemcpyDeviceToHost, s));
    PSM_CUDA_TRY(c->st, cudaStreamSynchronize(s));
    c->have_traces = c->traces_readable = false;  // the cube now holds the last residual
    if (resid)
        for (int k = 0; k <= iters; ++k) resid[k] = std::sqrt(std::max(h[k], 0.0));
    return read_device_error(c);
}

int psm_count_terms_rows(psm_ctx* c, int64_t* per_row) {
    if (!c || !per_row) return PSM_ERR_ARG;
    if (!c->have_geom || !c->have_vrms)
        return c->st.fail(PSM_ERR_STATE, "geometry and vrms must be set");
    cudaSetDevice(c->device);
    FwdParams P = volume_params(c);
    P.jobs = c->d_jobs_all.as<Job>();
    const size_t nj = c->jobs_all.size();
    PSM_CUDA_TRY(c->st, c->count.ensure(nj * sizeof(unsigned long long)));
    PSM_CUDA_TRY(c->st, cudaMemsetAsync(c->count.p, 0, nj * sizeof(unsigned long long),
                                        c->stream));
    psm::count_kernel<<<dim3(c->g.n_ox, static_cast<unsigned>(nj)), 256, 0, c->stream>>>(
        P, c->count.as<unsigned long long>());
    PSM_CUDA_TRY(c->st, cudaGetLastError());
    std::vector<unsigned long long> h(nj);
    PSM_CUDA_TRY(c->st, cudaMemcpyAsync(h.data(), c->count.p, nj * sizeof(unsigned long long),
                                        cudaMemcpyDeviceToHost, c->stream));
    PSM_CUDA_TRY(c->st, cudaStreamSynchronize(c->stream));
    for (size_t j = 0; j < nj; ++j) per_row[c->jobs_all[j].row] = static_cast<int64_t>(h[j]);
    return PSM_OK;
}

int psm_count_terms(psm_ctx* c, int64_t* n_terms) {
    if (!c || !n_terms) return PSM_ERR_ARG;
    if (!c->have_geom) return c->st.fail(PSM_ERR_STATE, "psm_set_geometry first");
    std::vector<int64_t> rows(c->g.n_oi, 0);
    int r = psm_count_terms_rows(c, rows.data());
    if (r) return r;
    int64_t s = 0;
    for (int64_t v : rows) s += v;
    *n_terms = s;
    return PSM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------- slabs

namespace {

// Centre (real inline) of output inline o (main.cpp:258-288).
inline int slab_center(const psm_geom& g, const int32_t* out_center, int o) {
    return out_center ? out_center[o] : std::min(std::max(o - g.pad_il, 0), g.n_il - 1);
}

// Input inlines [lo, hi) output inline o reads (migration_kernel.cpp:404-409).
inline void slab_reads(const psm_geom& g, const int32_t* out_center, int o, int* lo, int* hi) {
    const int c = slab_center(g, out_center, o);
    *lo = std::max(0, c - g.m_il - g.pad_il);
    *hi = std::min(g.n_il, c + g.m_il + 1 + g.pad_il);
}

bool slab_args_ok(const psm_geom* g, const int32_t* out_center) {
    std::string why;
    if (!g || check_geometry(*g, &why) != PSM_OK) return false;
    for (int o = 0; out_center && o < g->n_oi; ++o)
        if (out_center[o] < 0 || out_center[o] >= g->n_il) return false;
    return true;
}

// The input range of output inlines [o0, o1): the union of their reads (centres need not be
// monotone when out_center is given).
void slab_range(const psm_geom& g, const int32_t* out_center, psm_slab* s) {
    s->i0 = g.n_il;
    s->i1 = 0;
    for (int o = s->o0; o < s->o1; ++o) {
        int lo, hi;
        slab_reads(g, out_center, o, &lo, &hi);
        s->i0 = std::min(s->i0, lo);
        s->i1 = std::max(s->i1, hi);
    }
}

}  // namespace

extern "C" {

int64_t psm_slab_bytes(const psm_geom* g, int32_t n_in, int32_t n_out) {
    if (!g || n_in < 0 || n_out < 0) return -1;
    const int64_t ns = trace_stride(g->n_t);
    const int64_t stage = store_of(g->precision) == psm::kStoreF32 ? 8 : 4;
    const int64_t per_trace = ns * (4 + 8) + (stage == 4 ? ns * 4 + 4 : 0) + 4LL * g->n_t;
    return int64_t(n_in) * g->n_xl * per_trace + int64_t(n_out) * g->n_ox * g->n_t * 4 +
           (int64_t(n_out) + n_in) * 64 + 4LL * g->n_t;
}

int psm_plan_slabs(const psm_geom* g, const int32_t* out_center, int64_t max_device_bytes,
                   psm_slab* slabs, int32_t max_slabs, int32_t* n_slabs) {
    if (!slab_args_ok(g, out_center) || !slabs || max_slabs <= 0 || !n_slabs) return PSM_ERR_ARG;
    int32_t n = 0;
    int o = 0;
    while (o < g->n_oi) {
        psm_slab s{o, o + 1, 0, 0};
        slab_range(*g, out_center, &s);
        if (max_device_bytes > 0 && psm_slab_bytes(g, s.i1 - s.i0, 1) > max_device_bytes)
            return PSM_ERR_UNSUPPORTED;
        while (s.o1 < g->n_oi) {  // grow while the next output inline still fits
            psm_slab t{s.o0, s.o1 + 1, 0, 0};
            slab_range(*g, out_center, &t);
            if (max_device_bytes > 0 &&
                psm_slab_bytes(g, t.i1 - t.i0, t.o1 - t.o0) > max_device_bytes)
                break;
            s = t;
        }
        if (n == max_slabs) return PSM_ERR_ARG;
        slabs[n++] = s;
        o = s.o1;
    }
    *n_slabs = n;
    return PSM_OK;
}

int psm_split_slabs(const psm_geom* g, const int32_t* out_center, const double* weight,
                    int32_t n_parts, psm_slab* slabs) {
    if (!slab_args_ok(g, out_center) || n_parts <= 0 || !slabs) return PSM_ERR_ARG;
    double total = 0.0;
    for (int o = 0; o < g->n_oi; ++o) total += weight ? std::max(weight[o], 0.0) : 1.0;
    int o = 0;
    double acc = 0.0;
    for (int32_t k = 0; k < n_parts; ++k) {
        psm_slab s{o, o, 0, 0};
        const double target = total * (k + 1) / n_parts;
        // take output inlines while the running work stays closest to the k-th quantile
        while (s.o1 < g->n_oi) {
            const double w = weight ? std::max(weight[s.o1], 0.0) : 1.0;
            if (k == n_parts - 1 || acc + w <= target || acc + 0.5 * w <= target) {
                acc += w;
                ++s.o1;
            } else {
                break;
            }
        }
        slab_range(*g, out_center, &s);
        if (s.o1 == s.o0) s.i0 = s.i1 = 0;
        slabs[k] = s;
        o = s.o1;
    }
    return PSM_OK;
}

int psm_slab_geometry(const psm_geom* g, const int32_t* out_center, const psm_slab* s,
                      psm_geom* local, int32_t* local_center) {
    if (!slab_args_ok(g, out_center) || !s || !local || !local_center) return PSM_ERR_ARG;
    if (s->o0 < 0 || s->o1 > g->n_oi || s->o0 >= s->o1) return PSM_ERR_ARG;
    psm_slab need{s->o0, s->o1, 0, 0};
    slab_range(*g, out_center, &need);
    if (s->i0 < 0 || s->i1 > g->n_il || s->i0 > need.i0 || s->i1 < need.i1) return PSM_ERR_ARG;
    *local = *g;
    local->n_il = s->i1 - s->i0;
    local->n_oi = s->o1 - s->o0;
    for (int o = s->o0; o < s->o1; ++o)
        local_center[o - s->o0] = slab_center(*g, out_center, o) - s->i0;
    return PSM_OK;
}

int psm_forward_streamed(psm_ctx* c, const psm_geom* g, const int32_t* out_center,
                         const float* traces, const float* vrms, float* image,
                         int64_t max_device_bytes) {
    if (!c || !traces || !vrms || !image) return PSM_ERR_ARG;
    if (!slab_args_ok(g, out_center)) return c->st.fail(PSM_ERR_ARG, "invalid geometry");
    std::vector<psm_slab> slabs(static_cast<size_t>(g->n_oi));
    int32_t n = 0;
    int rc = psm_plan_slabs(g, out_center, max_device_bytes, slabs.data(), g->n_oi, &n);
    if (rc) return c->st.fail(rc, "one output inline exceeds the device budget");
    cudaSetDevice(c->device);
    const size_t trace = static_cast<size_t>(g->n_xl) * g->n_t;  // floats of one inline
    const size_t row = static_cast<size_t>(g->n_ox) * g->n_t;    // floats of one output inline
    const size_t per_il_tr = static_cast<size_t>(g->n_xl);
    const int ns = trace_stride(g->n_t);
    // Consecutive slabs' input inlines overlap (each output inline reads about m_il + pad_il
    // inlines either side), so the device window rolls: the inlines the next slab shares with
    // this one stay on the device (pair cube or 16-bit words, and Vrms), moved to the front of
    // their buffers, and only the new inlines are uploaded and prepared.  The new inlines of
    // slab k + 1 go up into a staging area while slab k migrates, and slab k's image returns
    // to the host while slab k + 1 migrates (two image buffers in turn), so the copies hide
    // behind the kernels.  A slab uploaded whole (the first) goes through psm_forward_host's
    // pipeline: its output inlines migrate as soon as their inputs are up, and their image
    // rows go straight to the host.  The raw traces of the kept inlines are not kept: after this call
    // the ctx holds the last slab's geometry and no readable traces.
    std::vector<psm_geom> loc(static_cast<size_t>(n));
    std::vector<std::vector<int32_t>> lcs(static_cast<size_t>(n));
    std::vector<int> keep(static_cast<size_t>(n), 0);  // inlines shared with the slab before
    int wide = 0, max_oi = 0, max_fresh = 0;
    for (int32_t k = 0; k < n; ++k) {
        const psm_slab& sl = slabs[k];
        lcs[k].resize(static_cast<size_t>(sl.o1 - sl.o0));
        if ((rc = psm_slab_geometry(g, out_center, &sl, &loc[k], lcs[k].data()))) return rc;
        if (sl.i1 - sl.i0 > slabs[wide].i1 - slabs[wide].i0) wide = k;
        max_oi = std::max(max_oi, sl.o1 - sl.o0);
        if (k > 0 && sl.i0 >= slabs[k - 1].i0 && sl.i0 < slabs[k - 1].i1)
            keep[k] = std::min(slabs[k - 1].i1, sl.i1) - sl.i0;
        if (k > 0 && keep[k] > 0) max_fresh = std::max(max_fresh, (sl.i1 - sl.i0) - keep[k]);
    }
    // size the device buffers for the widest slab once, so that none regrows
    if (n > 1 && (rc = psm_set_geometry(c, &loc[wide], lcs[wide].data()))) return rc;
    for (cudaStream_t* t : {&c->copy_stream, &c->d2h_stream})
        if (!*t) PSM_CUDA_TRY(c->st, cudaStreamCreateWithFlags(t, cudaStreamNonBlocking));
    for (cudaEvent_t* e : {&c->ev_placed, &c->ev_staged, &c->ev_done[0], &c->ev_done[1]})
        if (!*e) PSM_CUDA_TRY(c->st, cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    const size_t fresh_rows = static_cast<size_t>(std::max(max_fresh, 1)) * per_il_tr;
    PSM_CUDA_TRY(c->st, c->str_tr.ensure(fresh_rows * ns * sizeof(float)));
    PSM_CUDA_TRY(c->st, c->str_v.ensure(fresh_rows * g->n_t * sizeof(float)));
    for (DevBuf& b : c->str_img)
        PSM_CUDA_TRY(c->st, b.ensure(static_cast<size_t>(max_oi) * row * sizeof(float)));
    // the staged rows' tail samples (n_t .. ns - 1) stay zero, as in the resident cube
    PSM_CUDA_TRY(c->st, cudaMemsetAsync(c->str_tr.p, 0, fresh_rows * ns * sizeof(float),
                                        c->stream));
    bool staged = false;  // the next slab's new inlines are in the staging area
    auto fresh_of = [&](int k) { return (slabs[k].i1 - slabs[k].i0) - keep[k]; };
    // stage slab k's new inlines (once the previous placement has read the staging area)
    auto stage = [&](int k) -> int {
        if (k >= n || keep[k] <= 0) return PSM_OK;
        if (fresh_of(k) > 0) {
            const int kp = keep[k], fresh = fresh_of(k);
            const size_t first = static_cast<size_t>(slabs[k].i0 + kp);
            PSM_CUDA_TRY(c->st, cudaStreamWaitEvent(c->copy_stream, c->ev_placed, 0));
            PSM_CUDA_TRY(c->st, upload_rows(c->staging, c->str_tr.p, ns * sizeof(float),
                                            traces + first * trace, g->n_t * sizeof(float),
                                            static_cast<size_t>(fresh) * per_il_tr,
                                            c->copy_stream));
            PSM_CUDA_TRY(c->st, upload(c->staging, c->str_v.p, vrms + first * trace,
                                       fresh * trace * sizeof(float), c->copy_stream));
            PSM_CUDA_TRY(c->st, cudaEventRecord(c->ev_staged, c->copy_stream));
        }
        staged = true;  // (nothing new to stage when fresh_of(k) is 0)
        return PSM_OK;
    };
    // slabs whose image rows went straight to the host (uploaded whole, in waves)
    std::vector<char> direct(static_cast<size_t>(n), 0);
    for (int32_t k = 0; k < n; ++k) {
        const psm_slab& sl = slabs[k];
        // a buffer that set_geometry had to grow was reallocated (its size changed), and
        // its contents are gone
        const DevBuf* bufs[4] = {&c->pairs, &c->words, &c->scales, &c->vrms};
        size_t sizes[4];
        for (int i = 0; i < 4; ++i) sizes[i] = bufs[i]->bytes;
        const bool had = k > 0 && c->have_traces && c->have_vrms;
        // (waits for slab k - 1's kernel: psm_set_geometry synchronises the stream)
        if ((rc = psm_set_geometry(c, &loc[k], lcs[k].data()))) return rc;
        bool same_bufs = true;
        for (int i = 0; i < 4; ++i)
            if ((i == 0 || i == 3 || c->store != psm::kStoreF32) && bufs[i]->bytes != sizes[i])
                same_bufs = false;
        if (!(had && same_bufs && keep[k] > 0 && staged)) {
            // the whole slab, uploaded in inline blocks: each output inline migrates once its
            // inputs are up, and its image rows go straight to the host; the next slab's new
            // inlines are staged while the last waves migrate
            staged = false;
            if (k > 0 && (rc = read_device_error(c))) return rc;  // (forward_waves clears it)
            if ((rc = forward_waves(c, traces + sl.i0 * trace, vrms + sl.i0 * trace,
                                    image + sl.o0 * row, [&] { return stage(k + 1); })))
                return rc;
            direct[k] = 1;
        } else {
            const int shift = sl.i0 - slabs[k - 1].i0;  // inlines
            const int kp = keep[k];
            // move kept inlines to the front, front to back in chunks of at most `shift`
            // inlines so that no copy overlaps itself
            auto move = [&](void* base, size_t il_bytes) -> cudaError_t {
                char* b = static_cast<char*>(base);
                for (int a = 0; shift > 0 && a < kp; a += shift) {
                    const int ch = std::min(shift, kp - a);
                    cudaError_t e = cudaMemcpyAsync(b + a * il_bytes, b + (a + shift) * il_bytes,
                                                    ch * il_bytes, cudaMemcpyDeviceToDevice,
                                                    c->stream);
                    if (e != cudaSuccess) return e;
                }
                return cudaSuccess;
            };
            if (c->store == psm::kStoreF32) {
                PSM_CUDA_TRY(c->st, move(c->pairs.p, per_il_tr * ns * sizeof(float2)));
            } else {
                PSM_CUDA_TRY(c->st, move(c->words.p, per_il_tr * ns * sizeof(uint32_t)));
                PSM_CUDA_TRY(c->st, move(c->scales.p, per_il_tr * sizeof(float)));
            }
            PSM_CUDA_TRY(c->st, move(c->vrms.p, trace * sizeof(float)));
            const int fresh = fresh_of(k);  // new inlines, after the kept ones, from staging
            if (fresh > 0) {
                const size_t r0 = static_cast<size_t>(kp) * per_il_tr;
                const size_t rows = static_cast<size_t>(fresh) * per_il_tr;
                PSM_CUDA_TRY(c->st, cudaStreamWaitEvent(c->stream, c->ev_staged, 0));
                if (c->store == psm::kStoreF32)
                    PSM_CUDA_TRY(c->st, build_pairs(c->str_tr.as<float>(),
                                                    c->pairs.as<float2>() + r0 * ns, rows, ns,
                                                    c->stream));
                else
                    PSM_CUDA_TRY(c->st, quantize(c->str_tr.as<float>(),
                                                 c->words.as<uint32_t>() + r0 * ns,
                                                 c->scales.as<float>() + r0, rows, ns, c->store,
                                                 c->stream));
                PSM_CUDA_TRY(c->st, cudaMemcpyAsync(c->vrms.as<float>() + kp * trace,
                                                    c->str_v.p, fresh * trace * sizeof(float),
                                                    cudaMemcpyDeviceToDevice, c->stream));
            }
            c->have_traces = c->have_vrms = true;
            c->traces_readable = false;  // the raw cube rows were not moved
        }
        if (!direct[k]) {  // migrate slab k into image buffer k % 2
            staged = false;
            PSM_CUDA_TRY(c->st, cudaEventRecord(c->ev_placed, c->stream));  // staging free again
            if (k == 0) PSM_CUDA_TRY(c->st, cudaMemsetAsync(c->err.p, 0, sizeof(int), c->stream));
            float* img = c->str_img[k & 1].as<float>();
            FwdParams P = volume_params(c);
            P.image = img;
            PSM_CUDA_TRY(c->st, launch_fwd(P, static_cast<int>(c->jobs.size()),
                                           c->g.amp_correction != 0, c->variant, c->stream,
                                           c->store, c->g.compensated != 0));
            PSM_CUDA_TRY(c->st, copy_rows(c, img, c->stream));  // padded inlines
            PSM_CUDA_TRY(c->st, cudaEventRecord(c->ev_done[k & 1], c->stream));
        }
        // while slab k migrates: stage the next slab's new inlines ...
        if (!direct[k] && (rc = stage(k + 1))) return rc;
        // ... and return slab k - 1's image
        if (k > 0 && !direct[k - 1]) {
            const psm_slab& pv = slabs[k - 1];
            PSM_CUDA_TRY(c->st, cudaStreamWaitEvent(c->d2h_stream, c->ev_done[(k - 1) & 1], 0));
            PSM_CUDA_TRY(c->st, download(c->staging, image + pv.o0 * row,
                                         c->str_img[(k - 1) & 1].p,
                                         (pv.o1 - pv.o0) * row * sizeof(float), c->d2h_stream));
            PSM_CUDA_TRY(c->st, cudaStreamSynchronize(c->d2h_stream));
        }
    }
    if (n > 0 && !direct[n - 1]) {
        const psm_slab& pv = slabs[n - 1];
        PSM_CUDA_TRY(c->st, download(c->staging, image + pv.o0 * row, c->str_img[(n - 1) & 1].p,
                                     (pv.o1 - pv.o0) * row * sizeof(float), c->stream));
    }
    PSM_CUDA_TRY(c->st, cudaStreamSynchronize(c->copy_stream));
    return read_device_error(c);
}

}  // extern "C"

// ---------------------------------------------------------------------------- batched launch

namespace {

struct BatchCube {
    const float* host = nullptr;
    int n_il = 0, n_xl = 0, n_t = 0, ns = 0;
    DevBuf data, pairs, words, scales;
};

struct BatchProblem {
    psm_problem src{};
    int cube = 0;
    std::vector<Job> jobs, jobs_all;
    std::vector<std::pair<int, int>> copies;
    DevBuf vrms, image, d_jobs, d_jobs_all, t0;
    FwdParams P{};
};

}  // namespace

struct psm_batch {
    psm_ctx* ctx = nullptr;
    std::vector<BatchCube> cubes;
    std::vector<BatchProblem> probs;
    int store = psm::kStoreF32;
    bool amp = true, kahan = false;
    int variant = PSM_FWD_DEFAULT;
    int mode = PSM_BATCH_PERSISTENT;
    int max_inl = 1, stage_cap = 0;
    int max_ns = 0;  // longest trace stride over the problems
    int grid = 1;  // persistent CTAs
    int order = PSM_ORDER_DEPTH_FIRST;
    // tile lists [time tile 128 / 256 / 512 samples (4 / 8 / 16 blocks a lane)][order]
    int n_items[6] = {0, 0, 0, 0, 0, 0};
    DevBuf items[6];
    std::unique_ptr<psm::BatchParams> params;  // every problem's FwdParams (kernel argument)
    DevBuf counter, il_pos;
    cudaGraphExec_t exec = nullptr;
    int exec_key = -1;  // variant and order the graph was captured with
    int64_t n_terms = -1;
    ~psm_batch() {
        if (exec) cudaGraphExecDestroy(exec);
    }
};

namespace {

// The tile list of a kernel whose time tile is 32 J samples, in the given order.
constexpr int item_list(int J, int order) { return 2 * (J == 4 ? 0 : (J == 8 ? 1 : 2)) + order; }
static_assert(item_list(4, 1) == 1 && item_list(8, 0) == 2 && item_list(16, 1) == 5,
              "tile list index");

// Shared-memory attribute and persistent grid (resident CTAs on every SM) of the batch
// kernel K; done before a stream capture, so the graph holds only the launch.
// Stage capacity of the persistent kernel K: the batch's (48 KB stages, or one whole trace),
// or for a kernel built for 3 CTAs per SM 32 KB stages, so that three CTAs fit an SM.
template <class K>
int persistent_stage_cap(const psm_batch& b) {
    if constexpr (K::MINB > 2) return std::max(stage_cap_for(K::MINB, K::STORE), b.max_ns);
    return b.stage_cap;
}

template <class K>
cudaError_t prepare_persistent(K, psm_batch& b) {
    auto* kern = psm::fwd_batch_kernel<K::AMP, K::PACKED, K::GB, K::J, K::STORE, K::KAHAN,
                                       K::PAIRS, K::MINB>;
    const size_t smem =
        psm::smem_layout(b.max_inl, persistent_stage_cap<K>(b), psm::store_bytes(K::STORE))
            .total;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    int per_sm = 0, n_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * (psm::kTX + 1), smem);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, b.ctx->device);
    if (e != cudaSuccess) return e;
    const int w = item_list(K::J, b.order);
    b.grid = std::max(1, std::min(b.n_items[w], n_sm * std::max(per_sm, 1)));
    return cudaSuccess;
}

template <class K>
cudaError_t launch_persistent(K, const psm_batch& b, cudaStream_t s) {
    auto* kern = psm::fwd_batch_kernel<K::AMP, K::PACKED, K::GB, K::J, K::STORE, K::KAHAN,
                                       K::PAIRS, K::MINB>;
    const int cap = persistent_stage_cap<K>(b);
    const size_t smem = psm::smem_layout(b.max_inl, cap, psm::store_bytes(K::STORE)).total;
    const int w = item_list(K::J, b.order);
    const psm::BatchParams* params = b.params.get();
    std::unique_ptr<psm::BatchParams> small;
    if constexpr (K::MINB > 2) {  // every problem stages into the smaller stages
        small = std::make_unique<psm::BatchParams>(*b.params);
        for (size_t i = 0; i < b.probs.size(); ++i) small->p[i].stage_cap = cap;
        params = small.get();
    }
    kern<<<b.grid, 32 * (psm::kTX + 1), smem, s>>>(
        *params, b.items[w].as<psm::BatchItem>(), b.n_items[w], b.counter.as<int>(),
        b.ctx->err.as<int>(), b.max_inl, cap);
    return cudaGetLastError();
}

// The one-grid kernel K (a CTA per tile of the list): its shared-memory attribute, set before
// a stream capture.
template <class K>
cudaError_t prepare_items(K, const psm_batch& b) {
    auto* kern = psm::fwd_items_kernel<K::AMP, K::PACKED, K::GB, K::J, K::STORE, K::KAHAN,
                                       K::PAIRS, K::MINB>;
    const size_t smem =
        psm::smem_layout(b.max_inl, persistent_stage_cap<K>(b), psm::store_bytes(K::STORE))
            .total;
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(smem));
}

template <class K>
cudaError_t launch_items(K, const psm_batch& b, cudaStream_t s) {
    auto* kern = psm::fwd_items_kernel<K::AMP, K::PACKED, K::GB, K::J, K::STORE, K::KAHAN,
                                       K::PAIRS, K::MINB>;
    const int cap = persistent_stage_cap<K>(b);
    const size_t smem = psm::smem_layout(b.max_inl, cap, psm::store_bytes(K::STORE)).total;
    const int w = item_list(K::J, b.order);
    if (b.n_items[w] <= 0) return cudaSuccess;
    const psm::BatchParams* params = b.params.get();
    std::unique_ptr<psm::BatchParams> small;
    if constexpr (K::MINB > 2) {  // every problem stages into the smaller stages
        small = std::make_unique<psm::BatchParams>(*b.params);
        for (size_t i = 0; i < b.probs.size(); ++i) small->p[i].stage_cap = cap;
        params = small.get();
    }
    kern<<<b.n_items[w], 32 * (psm::kTX + 1), smem, s>>>(
        *params, b.items[w].as<psm::BatchItem>(), b.max_inl, cap);
    return cudaGetLastError();
}

// Repeated output rows of every problem (padded output inlines, main.cpp:268-285).
cudaError_t batch_copies(const psm_batch& b, cudaStream_t s) {
    for (const BatchProblem& p : b.probs) {
        const size_t row = static_cast<size_t>(p.src.geom.n_ox) * p.src.geom.n_t;
        for (const auto& cp : p.copies) {
            cudaError_t e = cudaMemcpyAsync(p.image.as<float>() + cp.first * row,
                                            p.image.as<float>() + cp.second * row,
                                            row * sizeof(float), cudaMemcpyDeviceToDevice, s);
            if (e != cudaSuccess) return e;
        }
    }
    return cudaSuccess;
}

// The work of one batched run, enqueued on s (persistent: counter and error word reset, one
// launch, row copies).
cudaError_t batch_enqueue(psm_batch& b, int variant, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(b.ctx->err.p, 0, sizeof(int), s);
    if (e != cudaSuccess) return e;
    if (b.mode == PSM_BATCH_ONE_GRID) {
        e = with_kernel(b.amp, variant, b.store, b.kahan,
                        [&](auto k) { return launch_items(k, b, s); });
        if (e != cudaSuccess) return e;
    } else if (b.mode == PSM_BATCH_PER_PROBLEM) {
        for (const BatchProblem& p : b.probs) {
            e = launch_fwd(p.P, static_cast<int>(p.jobs.size()), b.amp, variant, s, b.store,
                           b.kahan);
            if (e != cudaSuccess) return e;
        }
    } else {
        e = cudaMemsetAsync(b.counter.p, 0, sizeof(int), s);
        if (e != cudaSuccess) return e;
        e = with_kernel(b.amp, variant, b.store, b.kahan,
                        [&](auto k) { return launch_persistent(k, b, s); });
        if (e != cudaSuccess) return e;
    }
    return batch_copies(b, s);
}

// Capture the run (either mode) into a CUDA graph once per variant, order and mode, then
// replay it.
int batch_launch(psm_batch* b) {
    psm_ctx* c = b->ctx;
    const int v = effective_variant(b->variant, b->store, b->kahan);
    const int key = (v * 2 + b->order) * 3 + b->mode;
    if (!b->exec || b->exec_key != key) {
        if (b->exec) {
            cudaGraphExecDestroy(b->exec);
            b->exec = nullptr;
        }
        if (b->mode == PSM_BATCH_ONE_GRID)
            PSM_CUDA_TRY(c->st, with_kernel(b->amp, v, b->store, b->kahan, [&](auto k) {
                             return prepare_items(k, *b);
                         }));
        else if (b->mode == PSM_BATCH_PERSISTENT)
            PSM_CUDA_TRY(c->st, with_kernel(b->amp, v, b->store, b->kahan, [&](auto k) {
                             return prepare_persistent(k, *b);
                         }));
        else {  // grid launches: the shared-memory attribute is set outside the capture
            size_t smem = 0;
            for (const BatchProblem& p : b->probs) smem = std::max(smem, fwd_smem(p.P, b->store));
            PSM_CUDA_TRY(c->st, with_kernel(b->amp, v, b->store, b->kahan,
                                            [&](auto k) { return prepare_grid(k, smem); }));
        }
        cudaGraph_t graph = nullptr;
        PSM_CUDA_TRY(c->st, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        const cudaError_t e = batch_enqueue(*b, v, c->stream);
        const cudaError_t e2 = cudaStreamEndCapture(c->stream, &graph);
        PSM_CUDA_TRY(c->st, e);
        PSM_CUDA_TRY(c->st, e2);
        const cudaError_t e3 = cudaGraphInstantiate(&b->exec, graph, 0);
        cudaGraphDestroy(graph);
        PSM_CUDA_TRY(c->st, e3);
        b->exec_key = key;
    }
    PSM_CUDA_TRY(c->st, cudaGraphLaunch(b->exec, c->stream));
    return PSM_OK;
}

// Upload (or re-upload) every cube and Vrms from the host arrays.
int batch_upload(psm_batch* b) {
    psm_ctx* c = b->ctx;
    cudaStream_t s = c->stream;
    for (BatchCube& q : b->cubes) {
        const size_t n_tr = static_cast<size_t>(q.n_il) * q.n_xl;
        PSM_CUDA_TRY(c->st, upload_rows(c->staging, q.data.p, q.ns * sizeof(float), q.host,
                                        q.n_t * sizeof(float), n_tr, s));
        if (b->store == psm::kStoreF32)
            PSM_CUDA_TRY(c->st, build_pairs(q.data.as<float>(), q.pairs.as<float2>(), n_tr,
                                            q.ns, s));
        else
            PSM_CUDA_TRY(c->st, quantize(q.data.as<float>(), q.words.as<uint32_t>(),
                                         q.scales.as<float>(), n_tr, q.ns, b->store, s));
    }
    for (BatchProblem& p : b->probs) {
        const psm_geom& g = p.src.geom;
        if (p.src.vrms_kind == PSM_VRMS_CUBE) {
            PSM_CUDA_TRY(c->st, upload(c->staging, p.vrms.p, p.src.vrms,
                                       static_cast<size_t>(g.n_il) * g.n_xl * g.n_t *
                                           sizeof(float),
                                       s));
        } else if (p.src.vrms_kind == PSM_VRMS_TRACE) {
            PSM_CUDA_TRY(c->st, cudaMemcpyAsync(p.vrms.p, p.src.vrms, g.n_t * sizeof(float),
                                                cudaMemcpyHostToDevice, s));
        }
    }
    return PSM_OK;
}

}  // namespace

extern "C" {

int psm_batch_create(psm_ctx* c, const psm_problem* problems, int n, psm_batch** out) {
    if (!c || !problems || n <= 0 || !out) return PSM_ERR_ARG;
    *out = nullptr;
    if (n > psm::kMaxBatchProblems)
        return c->st.fail(PSM_ERR_UNSUPPORTED, "at most " +
                                                   std::to_string(psm::kMaxBatchProblems) +
                                                   " problems per batch");
    cudaSetDevice(c->device);
    std::unique_ptr<psm_batch> b(new (std::nothrow) psm_batch());
    if (!b) return PSM_ERR_NOMEM;
    b->ctx = c;
    b->probs.resize(n);
    const psm_geom& g0 = problems[0].geom;
    b->store = store_of(g0.precision);
    b->amp = g0.amp_correction != 0;
    b->kahan = g0.compensated != 0;
    int max_il = 1;
    for (int i = 0; i < n; ++i) {
        const psm_problem& src = problems[i];
        const psm_geom& g = src.geom;
        std::string why;
        int rc = check_geometry(g, &why);
        if (rc) return c->st.fail(rc, "problem " + std::to_string(i) + ": " + why);
        if ((g.amp_correction != 0) != b->amp || g.precision != g0.precision ||
            (g.compensated != 0) != b->kahan)
            return c->st.fail(PSM_ERR_ARG, "problems differ in amp_correction, precision or "
                                           "compensated");
        if (!src.traces || (src.vrms_kind != PSM_VRMS_CONSTANT && !src.vrms) ||
            src.vrms_kind < PSM_VRMS_CUBE || src.vrms_kind > PSM_VRMS_CONSTANT ||
            (src.vrms_kind == PSM_VRMS_CONSTANT && !(src.velocity >= 0.0f)))
            return c->st.fail(PSM_ERR_ARG, "problem " + std::to_string(i) +
                                               ": traces / vrms / velocity");
        BatchProblem& p = b->probs[i];
        p.src = src;
        if (!plan_jobs(g, src.out_center, p.jobs, p.jobs_all, p.copies))
            return c->st.fail(PSM_ERR_ARG, "problem " + std::to_string(i) +
                                               ": out_center out of range");
        // cube shared with an earlier problem given the same host array and grid
        int cube = -1;
        for (size_t k = 0; k < b->cubes.size(); ++k) {
            const BatchCube& q = b->cubes[k];
            if (q.host == src.traces && q.n_il == g.n_il && q.n_xl == g.n_xl && q.n_t == g.n_t)
                cube = static_cast<int>(k);
        }
        if (cube < 0) {
            cube = static_cast<int>(b->cubes.size());
            b->cubes.emplace_back();
            BatchCube& q = b->cubes.back();
            q.host = src.traces;
            q.n_il = g.n_il;
            q.n_xl = g.n_xl;
            q.n_t = g.n_t;
            q.ns = trace_stride(g.n_t);
        }
        p.cube = cube;
        max_il = std::max(max_il, g.n_il);
        b->max_inl = std::max(b->max_inl, max_inline_window(p.jobs_all));
        b->stage_cap = std::max(b->stage_cap, stage_cap(trace_stride(g.n_t), b->store));
        b->max_ns = std::max(b->max_ns, trace_stride(g.n_t));
    }
    if (psm::smem_layout(b->max_inl, b->stage_cap, psm::store_bytes(b->store)).total >
        kMaxDynSmem)
        return c->st.fail(PSM_ERR_UNSUPPORTED, "problems too large for one staging ring");
    cudaStream_t s = c->stream;
    PSM_CUDA_TRY(c->st, c->err.ensure(sizeof(int)));
    for (BatchCube& q : b->cubes) {
        const size_t n = static_cast<size_t>(q.n_il) * q.n_xl * q.ns;
        PSM_CUDA_TRY(c->st, q.data.ensure(n * sizeof(float)));
        PSM_CUDA_TRY(c->st, cudaMemsetAsync(q.data.p, 0, n * sizeof(float), s));
        if (b->store == psm::kStoreF32) {
            PSM_CUDA_TRY(c->st, q.pairs.ensure(n * sizeof(float2)));
        } else {
            PSM_CUDA_TRY(c->st, q.words.ensure(n * sizeof(uint32_t)));
            PSM_CUDA_TRY(c->st, q.scales.ensure(static_cast<size_t>(q.n_il) * q.n_xl *
                                                sizeof(float)));
        }
    }
    std::vector<int> pos(max_il);
    for (int i = 0; i < max_il; ++i) pos[i] = i;
    PSM_CUDA_TRY(c->st, b->il_pos.ensure(max_il * sizeof(int)));
    PSM_CUDA_TRY(c->st, cudaMemcpyAsync(b->il_pos.p, pos.data(), max_il * sizeof(int),
                                        cudaMemcpyHostToDevice, s));
    b->params.reset(new (std::nothrow) psm::BatchParams());
    if (!b->params) return PSM_ERR_NOMEM;
    std::vector<std::vector<float>> host_t0(n), host_v(n);
    for (int i = 0; i < n; ++i) {
        BatchProblem& p = b->probs[i];
        const psm_geom& g = p.src.geom;
        const BatchCube& q = b->cubes[p.cube];
        const int vk = p.src.vrms_kind;
        const size_t nv = vk == PSM_VRMS_CUBE ? static_cast<size_t>(g.n_il) * g.n_xl * g.n_t
                                              : static_cast<size_t>(g.n_t);
        PSM_CUDA_TRY(c->st, p.vrms.ensure(nv * sizeof(float)));
        PSM_CUDA_TRY(c->st, p.image.ensure(static_cast<size_t>(g.n_oi) * g.n_ox * g.n_t *
                                           sizeof(float)));
        PSM_CUDA_TRY(c->st, p.d_jobs.ensure(p.jobs.size() * sizeof(Job)));
        PSM_CUDA_TRY(c->st, p.d_jobs_all.ensure(p.jobs_all.size() * sizeof(Job)));
        PSM_CUDA_TRY(c->st, p.t0.ensure(g.n_t * sizeof(float)));
        host_t0[i].resize(g.n_t);
        for (int t = 0; t < g.n_t; ++t)
            host_t0[i][t] = static_cast<float>(static_cast<double>(t) * g.dt_seconds);
        PSM_CUDA_TRY(c->st, cudaMemcpyAsync(p.t0.p, host_t0[i].data(), g.n_t * sizeof(float),
                                            cudaMemcpyHostToDevice, s));
        PSM_CUDA_TRY(c->st, cudaMemcpyAsync(p.d_jobs.p, p.jobs.data(), p.jobs.size() * sizeof(Job),
                                            cudaMemcpyHostToDevice, s));
        PSM_CUDA_TRY(c->st, cudaMemcpyAsync(p.d_jobs_all.p, p.jobs_all.data(),
                                            p.jobs_all.size() * sizeof(Job),
                                            cudaMemcpyHostToDevice, s));
        if (vk == PSM_VRMS_CONSTANT) {
            host_v[i].assign(g.n_t, p.src.velocity);
            PSM_CUDA_TRY(c->st, cudaMemcpyAsync(p.vrms.p, host_v[i].data(), g.n_t * sizeof(float),
                                                cudaMemcpyHostToDevice, s));
        }
        FwdParams& P = p.P;
        P.pairs = q.pairs.as<float2>();
        P.words = q.words.as<uint32_t>();
        P.scales = q.scales.as<float>();
        P.vrms = p.vrms.as<float>();
        P.image = p.image.as<float>();
        P.jobs = p.d_jobs.as<Job>();
        P.il_pos = b->il_pos.as<int>();
        P.t0 = p.t0.as<float>();
        P.err = c->err.as<int>();
        P.wait_us = c->wait_us;
        P.fault = c->fault;
        P.compat_pad = g.compat_omp_pad != 0;
        P.n_ci = g.n_il;
        P.n_cx = g.n_xl;
        P.n_t = g.n_t;
        P.ns = q.ns;
        P.n_vx = g.n_xl;
        P.n_ox = g.n_ox;
        P.xoff = -g.pad_xl;
        P.max_inl = max_inline_window(p.jobs_all);
        P.stage_cap = stage_cap(q.ns, b->store);
        fill_consts(P, g.dt, g.d_il, g.d_xl, g.tan2_theta);
        if (vk != PSM_VRMS_CUBE) P.vs_x = P.vs_row = 0;  // one Vrms trace for every point
        b->params->p[i] = P;
    }
    // tile lists, for 128-, 256- and 512-sample time tiles, in two orders:
    //  * depth first: deepest time tiles first (the aperture, and so the work, grows with
    //    t0), then output inline, crossline tile and problem, so panels over one cube take
    //    the same tile one after another and the long tiles start early;
    //  * problem after problem, each in the grid kernel's order (crossline tile fastest,
    //    then output inline, then time tile, deepest first).
    PSM_CUDA_TRY(c->st, b->counter.ensure(sizeof(int)));
    for (int w = 0; w < 6; ++w) {
        const int TT = 32 * (4 << (w / 2));
        std::vector<psm::BatchItem> items;
        for (int i = 0; i < n; ++i) {
            const BatchProblem& p = b->probs[i];
            const psm_geom& g = p.src.geom;
            for (int T0 = (g.n_t - 1) / TT * TT; T0 >= 0; T0 -= TT)
                for (int j = 0; j < static_cast<int>(p.jobs.size()); ++j)
                    for (int x0 = 0; x0 < g.n_ox; x0 += psm::kTX) items.push_back({i, j, x0, T0});
        }
        if ((w & 1) == PSM_ORDER_DEPTH_FIRST)
            std::stable_sort(items.begin(), items.end(),
                             [](const psm::BatchItem& a, const psm::BatchItem& z) {
                                 if (a.T0 != z.T0) return a.T0 > z.T0;
                                 if (a.job != z.job) return a.job < z.job;
                                 if (a.x0 != z.x0) return a.x0 < z.x0;
                                 return a.prob < z.prob;
                             });
        b->n_items[w] = static_cast<int>(items.size());
        PSM_CUDA_TRY(c->st, b->items[w].ensure(items.size() * sizeof(psm::BatchItem)));
        PSM_CUDA_TRY(c->st, cudaMemcpyAsync(b->items[w].p, items.data(),
                                            items.size() * sizeof(psm::BatchItem),
                                            cudaMemcpyHostToDevice, s));
        PSM_CUDA_TRY(c->st, cudaStreamSynchronize(s));  // items is released next iteration
    }
    int rc = batch_upload(b.get());
    if (rc) return rc;
    PSM_CUDA_TRY(c->st, cudaStreamSynchronize(s));
    *out = b.release();
    return PSM_OK;
}

int psm_batch_destroy(psm_batch* b) {
    if (!b) return PSM_OK;
    cudaSetDevice(b->ctx->device);
    cudaStreamSynchronize(b->ctx->stream);
    delete b;
    return PSM_OK;
}

int psm_batch_reload(psm_batch* b) {
    if (!b) return PSM_ERR_ARG;
    cudaSetDevice(b->ctx->device);
    return batch_upload(b);
}

int psm_batch_get_mode(psm_batch* b, int* mode) {
    if (!b || !mode) return PSM_ERR_ARG;
    *mode = b->mode;
    return PSM_OK;
}

int psm_batch_set_mode(psm_batch* b, int mode) {
    if (!b || mode < PSM_BATCH_PERSISTENT || mode > PSM_BATCH_ONE_GRID)
        return PSM_ERR_ARG;
    b->mode = mode;
    return PSM_OK;
}

int psm_batch_set_order(psm_batch* b, int order) {
    if (!b || (order != PSM_ORDER_DEPTH_FIRST && order != PSM_ORDER_PROBLEM)) return PSM_ERR_ARG;
    b->order = order;
    return PSM_OK;
}

int psm_batch_get_order(psm_batch* b, int* order) {
    if (!b || !order) return PSM_ERR_ARG;
    *order = b->order;
    return PSM_OK;
}

int psm_batch_set_variant(psm_batch* b, int variant) {
    if (!b || variant < 0 || variant >= PSM_FWD_N_VARIANTS) return PSM_ERR_ARG;
    b->variant = variant;
    return PSM_OK;
}

int psm_batch_get_variant(psm_batch* b, int* variant) {
    if (!b || !variant) return PSM_ERR_ARG;
    *variant = effective_variant(b->variant, b->store, b->kahan);
    return PSM_OK;
}

int psm_batch_run_async(psm_batch* b) {
    if (!b) return PSM_ERR_ARG;
    cudaSetDevice(b->ctx->device);
    return batch_launch(b);
}

int psm_batch_synchronize(psm_batch* b) {
    if (!b) return PSM_ERR_ARG;
    return psm_synchronize(b->ctx);
}

int psm_batch_run(psm_batch* b) {
    int r = psm_batch_run_async(b);
    return r ? r : psm_batch_synchronize(b);
}

int psm_batch_autotune(psm_batch* b, float* ms, int* best, int* best_order, int* best_mode) {
    if (!b) return PSM_ERR_ARG;
    psm_ctx* c = b->ctx;
    cudaSetDevice(c->device);
    if (ms)
        for (int v = 0; v < 5 * PSM_FWD_N_VARIANTS; ++v) ms[v] = 0.0f;
    cudaEvent_t e0, e1;
    PSM_CUDA_TRY(c->st, cudaEventCreate(&e0));
    PSM_CUDA_TRY(c->st, cudaEventCreate(&e1));
    int pick = effective_variant(PSM_FWD_DEFAULT, b->store, b->kahan);
    int pick_order = b->order, pick_mode = b->mode;
    float pick_ms = 3.0e38f;
    int rc = PSM_OK;
    // schedules: persistent depth-first / problem order, one launch per problem, one grid
    // depth-first / problem order
    for (int sch = 0; sch < 5 && rc == PSM_OK; ++sch) {
        b->mode = sch < 2 ? PSM_BATCH_PERSISTENT
                          : (sch == 2 ? PSM_BATCH_PER_PROBLEM : PSM_BATCH_ONE_GRID);
        b->order = sch < 2 ? sch : (sch == 2 ? PSM_ORDER_DEPTH_FIRST : sch - 3);
        for (int v = 1; v < PSM_FWD_N_VARIANTS && rc == PSM_OK; ++v) {
            if (effective_variant(v, b->store, b->kahan) != v) continue;  // same kernel
            b->variant = v;
            float t = 0.0f;
            if ((rc = psm_batch_run(b)) != PSM_OK) break;  // warm: graph capture, first launch
            cudaEventRecord(e0, c->stream);
            if ((rc = batch_launch(b)) != PSM_OK) break;
            cudaEventRecord(e1, c->stream);
            if ((rc = psm_batch_synchronize(b)) != PSM_OK) break;
            cudaEventElapsedTime(&t, e0, e1);
            if (ms) ms[sch * PSM_FWD_N_VARIANTS + v] = t;
            if (t < pick_ms) {
                pick_ms = t;
                pick = v;
                pick_order = b->order;
                pick_mode = b->mode;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->variant = pick;
    b->order = pick_order;
    b->mode = pick_mode;
    if (rc == PSM_OK && best) *best = pick;
    if (rc == PSM_OK && best_order) *best_order = pick_order;
    if (rc == PSM_OK && best_mode) *best_mode = pick_mode;
    return rc;
}

int psm_batch_image_device(psm_batch* b, int i, float** dev) {
    if (!b || !dev || i < 0 || i >= static_cast<int>(b->probs.size())) return PSM_ERR_ARG;
    *dev = b->probs[i].image.as<float>();
    return PSM_OK;
}

int psm_batch_get_image(psm_batch* b, int i, float* image) {
    if (!b || !image || i < 0 || i >= static_cast<int>(b->probs.size())) return PSM_ERR_ARG;
    psm_ctx* c = b->ctx;
    cudaSetDevice(c->device);
    const psm_geom& g = b->probs[i].src.geom;
    PSM_CUDA_TRY(c->st, download(c->staging, image, b->probs[i].image.p,
                                 static_cast<size_t>(g.n_oi) * g.n_ox * g.n_t * sizeof(float),
                                 c->stream));
    PSM_CUDA_TRY(c->st, cudaStreamSynchronize(c->stream));
    return read_device_error(c);
}

int psm_batch_count_terms(psm_batch* b, int64_t* n_terms) {
    if (!b || !n_terms) return PSM_ERR_ARG;
    psm_ctx* c = b->ctx;
    cudaSetDevice(c->device);
    if (b->n_terms < 0) {
        size_t nj = 0;
        for (const BatchProblem& p : b->probs) nj += p.jobs_all.size();
        PSM_CUDA_TRY(c->st, c->count.ensure(nj * sizeof(unsigned long long)));
        PSM_CUDA_TRY(c->st, cudaMemsetAsync(c->count.p, 0, nj * sizeof(unsigned long long),
                                            c->stream));
        size_t off = 0;
        for (const BatchProblem& p : b->probs) {
            FwdParams P = p.P;
            P.jobs = p.d_jobs_all.as<Job>();
            psm::count_kernel<<<dim3(p.src.geom.n_ox, static_cast<unsigned>(p.jobs_all.size())),
                                256, 0, c->stream>>>(P, c->count.as<unsigned long long>() + off);
            PSM_CUDA_TRY(c->st, cudaGetLastError());
            off += p.jobs_all.size();
        }
        std::vector<unsigned long long> h(nj);
        PSM_CUDA_TRY(c->st, cudaMemcpyAsync(h.data(), c->count.p, nj * sizeof(unsigned long long),
                                            cudaMemcpyDeviceToHost, c->stream));
        PSM_CUDA_TRY(c->st, cudaStreamSynchronize(c->stream));
        int64_t s = 0;
        for (unsigned long long v : h) s += static_cast<int64_t>(v);
        b->n_terms = s;
    }
    *n_terms = b->n_terms;
    return PSM_OK;
}

}  // extern "C"

extern "C" {

// ---------------------------------------------------------------------------- per inline

namespace {
struct InlineStaging {
    int device = -1;
    cudaStream_t stream = nullptr;
    Status st;
    DevBuf data, pairs, vel, out, job, il_pos, t0, err;
    ~InlineStaging() {
        if (stream) cudaStreamDestroy(stream);
    }
};
thread_local std::unique_ptr<InlineStaging> tl_staging;
thread_local std::string tl_inline_error;
}  // namespace

int psm_kirchhoff_inline(const float* input_buffer, size_t n_buf_il, size_t n_buf_xl,
                         size_t n_t, const float* velocity_slice, float* output_slice,
                         size_t n_out_xl, const int32_t* il_pos_indices,
                         const int32_t* /*xl_pos_indices*/, int32_t current_il_pos,
                         int32_t current_xl_start, float dt, const float* t0_times,
                         float tan_theta_sq, float inline_bin_size,
                         float crossline_bin_size, int amp_correction) {
    tl_inline_error.clear();
    if (n_out_xl == 0 || n_t == 0) return PSM_OK;  // migration_kernel.cpp:35-37
    if (!output_slice || !t0_times || (n_buf_il && (!input_buffer || !il_pos_indices)) ||
        (n_buf_xl && !velocity_slice)) {
        tl_inline_error = "null pointer argument";
        return PSM_ERR_ARG;
    }
    if (n_buf_il > 0x7fffffff || n_buf_xl > 0x7fffffff || n_t > 0x7fffffff ||
        n_out_xl > 0x7fffffff) {
        tl_inline_error = "size too large";
        return PSM_ERR_ARG;
    }
    const int ns = trace_stride(static_cast<int>(n_t));
    if (psm::smem_layout(std::max<int>(static_cast<int>(n_buf_il), 1), stage_cap(ns)).total >
        kMaxDynSmem) {
        tl_inline_error = "n_t / buffer too large for the staging ring";
        return PSM_ERR_UNSUPPORTED;
    }
    if (!tl_staging) tl_staging.reset(new (std::nothrow) InlineStaging());
    InlineStaging* S = tl_staging.get();
    if (!S) return PSM_ERR_NOMEM;
    int dev = 0;
    cudaGetDevice(&dev);
    auto fail = [&](int code, const std::string& m) {
        tl_inline_error = m;
        return code;
    };
#define PSM_INL_TRY(call)                                                                   \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return fail(e_ == cudaErrorMemoryAllocation ? PSM_ERR_NOMEM : PSM_ERR_CUDA,     \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                \
    } while (0)
    if (S->device != dev || !S->stream) {
        if (S->stream) cudaStreamDestroy(S->stream);
        S->stream = nullptr;
        PSM_INL_TRY(cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking));
        S->device = dev;
    }
    const size_t n_tr = n_buf_il * n_buf_xl;
    PSM_INL_TRY(S->data.ensure(std::max<size_t>(n_tr, 1) * ns * sizeof(float)));
    PSM_INL_TRY(S->pairs.ensure(std::max<size_t>(n_tr, 1) * ns * sizeof(float2)));
    PSM_INL_TRY(S->vel.ensure(std::max<size_t>(n_buf_xl, 1) * n_t * sizeof(float)));
    PSM_INL_TRY(S->out.ensure(n_out_xl * n_t * sizeof(float)));
    PSM_INL_TRY(S->job.ensure(sizeof(Job)));
    PSM_INL_TRY(S->il_pos.ensure(std::max<size_t>(n_buf_il, 1) * sizeof(int)));
    PSM_INL_TRY(S->t0.ensure(n_t * sizeof(float)));
    PSM_INL_TRY(S->err.ensure(sizeof(int)));
    cudaStream_t s = S->stream;
    if (n_tr) {
        PSM_INL_TRY(cudaMemsetAsync(S->data.p, 0, n_tr * ns * sizeof(float), s));
        PSM_INL_TRY(cudaMemcpy2DAsync(S->data.p, ns * sizeof(float), input_buffer,
                                      n_t * sizeof(float), n_t * sizeof(float), n_tr,
                                      cudaMemcpyHostToDevice, s));
        PSM_INL_TRY(build_pairs(S->data.as<float>(), S->pairs.as<float2>(), n_tr, ns, s));
    }
    if (n_buf_xl)
        PSM_INL_TRY(cudaMemcpyAsync(S->vel.p, velocity_slice, n_buf_xl * n_t * sizeof(float),
                                    cudaMemcpyHostToDevice, s));
    if (n_buf_il)
        PSM_INL_TRY(cudaMemcpyAsync(S->il_pos.p, il_pos_indices, n_buf_il * sizeof(int),
                                    cudaMemcpyHostToDevice, s));
    PSM_INL_TRY(cudaMemcpyAsync(S->t0.p, t0_times, n_t * sizeof(float),
                                cudaMemcpyHostToDevice, s));
    // migration_kernel.cpp:48-49
    const int32_t cur = (current_il_pos >= 0 && current_il_pos < static_cast<int32_t>(n_buf_il))
                            ? il_pos_indices[current_il_pos]
                            : 0;
    Job j{0, 0, cur, 0, static_cast<int>(n_buf_il)};
    PSM_INL_TRY(cudaMemcpyAsync(S->job.p, &j, sizeof(Job), cudaMemcpyHostToDevice, s));
    PSM_INL_TRY(cudaMemsetAsync(S->err.p, 0, sizeof(int), s));
    FwdParams P{};
    P.pairs = S->pairs.as<float2>();
    P.vrms = S->vel.as<float>();
    P.image = S->out.as<float>();
    P.jobs = S->job.as<Job>();
    P.il_pos = S->il_pos.as<int>();
    P.t0 = S->t0.as<float>();
    P.err = S->err.as<int>();
    P.n_ci = static_cast<int>(n_buf_il);
    P.n_cx = static_cast<int>(n_buf_xl);
    P.n_t = static_cast<int>(n_t);
    P.ns = ns;
    P.n_vx = static_cast<int>(n_buf_xl);
    P.n_ox = static_cast<int>(n_out_xl);
    P.xoff = current_xl_start;
    P.max_inl = std::max<int>(static_cast<int>(n_buf_il), 1);
    P.stage_cap = stage_cap(ns);
    fill_consts(P, dt, inline_bin_size, crossline_bin_size, tan_theta_sq);
    for (size_t i = 1; i < n_buf_il; ++i)  // mirrored pairs need consecutive inline positions
        if (il_pos_indices[i] != il_pos_indices[i - 1] + 1) P.pairable = 0;
    PSM_INL_TRY(launch_fwd(P, 1, amp_correction != 0, PSM_FWD_DEFAULT, s));
    PSM_INL_TRY(cudaMemcpyAsync(output_slice, S->out.p, n_out_xl * n_t * sizeof(float),
                                cudaMemcpyDeviceToHost, s));
    int h = 0;
    PSM_INL_TRY(cudaMemcpyAsync(&h, S->err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    PSM_INL_TRY(cudaStreamSynchronize(s));
    if (h) return fail(PSM_ERR_DEVICE, "kernel reported device error flags " + std::to_string(h));
#undef PSM_INL_TRY
    return PSM_OK;
}

const char* psm_kirchhoff_inline_error(void) { return tl_inline_error.c_str(); }

}  // extern "C"

// ---------------------------------------------------------------------------- no allocation
//
// psm_forward_noalloc runs the forward kernel on caller-owned device buffers.  Its working
// memory (error word, job table, inline positions, time axis) lives in this one file-scope
// device array instead of cudaMalloc'd buffers.  On the host, g_noalloc_scratch names a
// host-side stand-in, not device memory: kernels only ever receive the address that
// cudaGetSymbolAddress returns for the current device.

namespace {

constexpr int kNoallocMaxRows = 4096;    // output inlines
constexpr int kNoallocMaxInl = 4096;     // input inlines
constexpr int kNoallocMaxT = 16384;      // samples per trace
constexpr size_t kNoallocErr = 0;        // int
constexpr size_t kNoallocJobs = 256;     // Job[kNoallocMaxRows]
constexpr size_t kNoallocPos = kNoallocJobs + ((sizeof(Job) * kNoallocMaxRows + 255) & ~size_t(255));
constexpr size_t kNoallocT0 = kNoallocPos + sizeof(int) * kNoallocMaxInl;
static_assert(kNoallocT0 + sizeof(float) * kNoallocMaxT <= PSM_NOALLOC_SCRATCH_BYTES,
              "no-allocation scratch layout exceeds its array");

__device__ __align__(256) unsigned char g_noalloc_scratch[PSM_NOALLOC_SCRATCH_BYTES];

constexpr int kNoallocMaxDevices = 64;
// Held for the whole of a psm_forward_noalloc call: it guards the per-device addresses and
// the host tables below, and serialises the calls of different host threads.
std::mutex g_noalloc_mutex;
unsigned char* g_noalloc_addr[kNoallocMaxDevices] = {};

// Host-side tables of a call (about 184 KB): static, so that a caller on a thread with a
// small stack can use the entry point; g_noalloc_mutex guards them.
struct NoallocTables {
    Job jobs[kNoallocMaxRows];
    int16_t first_row_of[kNoallocMaxInl];
    int16_t dup_dst[kNoallocMaxRows], dup_src[kNoallocMaxRows];
    int pos[kNoallocMaxInl];
    float t0[kNoallocMaxT];
};
NoallocTables g_noalloc_tables;

// Device address of g_noalloc_scratch on the current device (looked up once per device;
// the caller holds g_noalloc_mutex).
cudaError_t noalloc_scratch(unsigned char** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kNoallocMaxDevices) return cudaErrorInvalidDevice;
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_noalloc_addr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_noalloc_addr[dev];
    return cudaSuccess;
}

}  // namespace

extern "C" int psm_forward_noalloc(const psm_geom* g, const int32_t* out_center,
                                   const float* d_pairs, const float* d_vrms, float* d_image,
                                   void* stream) {
    if (!g || !d_pairs || !d_vrms || !d_image) return PSM_ERR_ARG;
    if (g->n_il <= 0 || g->n_xl <= 0 || g->n_t <= 0 || g->n_oi <= 0 || g->n_ox <= 0 ||
        g->pad_il < 0 || g->pad_xl < 0 || g->m_il < 0 || !(g->dt > 0.0f) ||
        !(g->d_il > 0.0f) || !(g->d_xl > 0.0f) || !(g->tan2_theta >= 0.0f) ||
        g->precision != PSM_F32 || g->compensated != 0 ||
        (reinterpret_cast<uintptr_t>(d_pairs) & 15u))
        return PSM_ERR_ARG;
    if (g->n_oi > kNoallocMaxRows || g->n_il > kNoallocMaxInl || g->n_t > kNoallocMaxT)
        return PSM_ERR_UNSUPPORTED;
    const int ns = trace_stride(g->n_t);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    NoallocTables& T = g_noalloc_tables;

    // jobs: one per distinct migrated inline, and the output rows that repeat it
    // (main.cpp:258-288, migration_kernel.cpp:404-409); fixed-size static tables, no heap
    Job* jobs = T.jobs;
    int16_t* first_row_of = T.first_row_of;
    int16_t *dup_dst = T.dup_dst, *dup_src = T.dup_src;
    int n_jobs = 0, n_dup = 0, max_inl = 1;
    for (int i = 0; i < g->n_il; ++i) first_row_of[i] = -1;
    for (int o = 0; o < g->n_oi; ++o) {
        const int cc = out_center ? out_center[o]
                                  : std::min(std::max(o - g->pad_il, 0), g->n_il - 1);
        if (cc < 0 || cc >= g->n_il) return PSM_ERR_ARG;
        const int rs = std::max(0, cc - g->m_il), re = std::min(g->n_il, cc + g->m_il + 1);
        Job j{o, cc, cc, std::max(0, rs - g->pad_il), std::min(g->n_il, re + g->pad_il)};
        max_inl = std::max(max_inl, j.i1 - j.i0);
        if (first_row_of[cc] < 0) {
            first_row_of[cc] = static_cast<int16_t>(o);
            jobs[n_jobs++] = j;
        } else {
            dup_dst[n_dup] = static_cast<int16_t>(o);
            dup_src[n_dup++] = first_row_of[cc];
        }
    }
    FwdParams P{};
    P.compat_pad = g->compat_omp_pad != 0;
    P.n_ci = g->n_il;
    P.n_cx = g->n_xl;
    P.n_t = g->n_t;
    P.ns = ns;
    P.n_vx = g->n_xl;
    P.n_ox = g->n_ox;
    P.xoff = -g->pad_xl;
    P.max_inl = max_inl;
    P.stage_cap = stage_cap(ns);
    if (!fwd_smem(P)) return PSM_ERR_UNSUPPORTED;
    fill_consts(P, g->dt, g->d_il, g->d_xl, g->tan2_theta);

    unsigned char* scratch = nullptr;
    if (noalloc_scratch(&scratch) != cudaSuccess) return PSM_ERR_CUDA;
    int* pos = T.pos;
    float* t0 = T.t0;
    for (int i = 0; i < g->n_il; ++i) pos[i] = i;
    for (int i = 0; i < g->n_t; ++i)
        t0[i] = static_cast<float>(static_cast<double>(i) * g->dt_seconds);  // main.cpp:216
#define PSM_NA_TRY(call)                                                            \
    do {                                                                            \
        if ((call) != cudaSuccess) return PSM_ERR_CUDA;                             \
    } while (0)
    // the array keeps the last call's contents: reset the error word, rewrite the tables
    PSM_NA_TRY(cudaMemsetAsync(scratch + kNoallocErr, 0, sizeof(int), s));
    PSM_NA_TRY(cudaMemcpyAsync(scratch + kNoallocJobs, jobs, sizeof(Job) * n_jobs,
                               cudaMemcpyHostToDevice, s));
    PSM_NA_TRY(cudaMemcpyAsync(scratch + kNoallocPos, pos, sizeof(int) * g->n_il,
                               cudaMemcpyHostToDevice, s));
    PSM_NA_TRY(cudaMemcpyAsync(scratch + kNoallocT0, t0, sizeof(float) * g->n_t,
                               cudaMemcpyHostToDevice, s));
    P.pairs = reinterpret_cast<const float2*>(d_pairs);
    P.vrms = d_vrms;
    P.image = d_image;
    P.jobs = reinterpret_cast<const Job*>(scratch + kNoallocJobs);
    P.il_pos = reinterpret_cast<const int*>(scratch + kNoallocPos);
    P.t0 = reinterpret_cast<const float*>(scratch + kNoallocT0);
    P.err = reinterpret_cast<int*>(scratch + kNoallocErr);
    PSM_NA_TRY(launch_fwd(P, n_jobs, g->amp_correction != 0, PSM_FWD_DEFAULT, s));
    const size_t row = static_cast<size_t>(g->n_ox) * g->n_t;
    for (int k = 0; k < n_dup; ++k)
        PSM_NA_TRY(cudaMemcpyAsync(d_image + dup_dst[k] * row, d_image + dup_src[k] * row,
                                   row * sizeof(float), cudaMemcpyDeviceToDevice, s));
    int h = 0;
    PSM_NA_TRY(cudaMemcpyAsync(&h, scratch + kNoallocErr, sizeof(int), cudaMemcpyDeviceToHost, s));
    PSM_NA_TRY(cudaStreamSynchronize(s));
#undef PSM_NA_TRY
    return h ? PSM_ERR_DEVICE : PSM_OK;
}
