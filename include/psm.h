/* psm.h -- C ABI of libpsm_cuda.so, the B200 (sm_100a) Kirchhoff post-stack 3D time
 * migration.
 *
 * The reference (sergeevsn/poststackmig3d) has no FFI; its seam is the static C++ class
 * MigrationKernel (include/migration_kernel.h:11-74), called from src/main.cpp:298, :314 and
 * :357.  The entry points below replace that seam.  Every function returns PSM_OK (0) or a
 * negative psm_status; no C++ exception crosses this boundary.  Host pointers are owned by
 * the caller; device memory allocated by the library is owned by the psm_ctx.  A psm_ctx is
 * bound to one device and one CUDA stream and is not thread-safe (one per host thread).
 * Calls return when their work is complete unless the name ends in _async.
 */
#ifndef PSM_H
#define PSM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    PSM_OK = 0,
    PSM_ERR_ARG = -1,        /* invalid argument / size */
    PSM_ERR_STATE = -2,      /* call out of order (e.g. forward before set_traces) */
    PSM_ERR_CUDA = -3,       /* a CUDA runtime call failed */
    PSM_ERR_NOMEM = -4,      /* device allocation failed */
    PSM_ERR_DEVICE = -5,     /* a kernel reported an error (bounded wait expired, ...) */
    PSM_ERR_UNSUPPORTED = -6 /* size or mode outside what the kernels handle */
} psm_status;

typedef enum { PSM_F32 = 0, PSM_BF16 = 1, PSM_F16 = 2 } psm_precision;

/* Geometry and migration parameters of a resident cube.  The values are the ones the
 * reference driver derives (src/main.cpp:124-217):
 *   n_il, n_xl, n_t   real input grid (sorted unique inline / crossline labels, samples)
 *   dt                sample interval in seconds, as float (main.cpp:363)
 *   dt_seconds        the same interval in double; t0[i] = float(i * dt_seconds)
 *                     (main.cpp:214-217)
 *   d_il, d_xl        inline_step / crossline_step in metres
 *   tan2_theta        float(tan(angle)) squared (main.cpp:188-189)
 *   m_il              inline aperture of the buffer (main.cpp:201)
 *   pad_il, pad_xl    inline_padding / crossline_padding
 *   n_oi, n_ox        output inlines / crosslines (labels padded by main.cpp:144-172)
 *   amp_correction    1/(t v^2) weighting on/off
 *   precision         storage of the traces in HBM (psm_precision): PSM_F32 keeps the
 *                     reference's fp32 samples; PSM_BF16 / PSM_F16 keep each trace as 16-bit
 *                     values d / scale with one fp32 scale per trace (scale = max |d|), and
 *                     sum in fp32.  No counterpart in the reference (fp32 only).
 *   compensated       nonzero: compensated (Kahan) summation over the aperture, partial
 *                     sums of at most 32 traces added with Kahan's compensation.  No
 *                     counterpart in the reference (plain fp32 sum, migration_kernel.cpp:229).
 *   compat_omp_pad    0: padded output crosslines have v = 0 and are zero, as in the
 *                     reference's serial build (migration_kernel.cpp:486-510).  Nonzero: the
 *                     trailing padded crosslines are migrated with the last real crossline's
 *                     Vrms (and their own position for r^2), which is what the reference's
 *                     OpenMP build computes (its per-sample caches, :60-72, are not reset for
 *                     crosslines with v = 0, and its nested crossline loop runs on one
 *                     thread, src/main.cpp:255); Vrms is taken to be positive.
 */
typedef struct {
    int32_t n_il, n_xl, n_t;
    int32_t pad_il, pad_xl;
    int32_t n_oi, n_ox;
    int32_t m_il;
    int32_t amp_correction;
    int32_t precision;
    float dt;
    float d_il, d_xl;
    float tan2_theta;
    double dt_seconds;
    int32_t compensated;
    int32_t compat_omp_pad;
} psm_geom;

typedef struct psm_ctx psm_ctx;

/* Library / device. */
const char *psm_version(void);
int psm_device_count(int *count);

/* Context lifetime: one GPU, one stream. */
int psm_create(psm_ctx **out, int device);
int psm_destroy(psm_ctx *ctx);
const char *psm_last_error(const psm_ctx *ctx); /* message of the last failure on ctx */

/* Geometry.  out_center[n_oi] gives, for every output inline, the real inline index it
 * migrates (main.cpp:258-288: padded output inlines take the nearest real inline); NULL
 * means the regular-label rule clamp(o - pad_il, 0, n_il - 1).  Replaces the per-inline
 * buffer set-up of MigrationKernel::prepareInputBufferWithPadding
 * (src/migration_kernel.cpp:385-468): the whole cube stays resident in HBM. */
int psm_set_geometry(psm_ctx *ctx, const psm_geom *g, const int32_t *out_center);

/* Upload the traces [n_il][n_xl][n_t] (host, float32, real grid, missing traces zero).
 * Replaces the per-inline re-reads of prepareInputBufferWithPadding. */
int psm_set_traces(psm_ctx *ctx, const float *data);

/* Upload the Vrms cube [n_il][n_xl][n_t] of the output points (host, float32).  Replaces
 * MigrationKernel::prepareVelocitySliceWithPadding (src/migration_kernel.cpp:470-511);
 * padded crosslines get v = 0 inside the kernel. */
int psm_set_vrms(psm_ctx *ctx, const float *vrms);

/* Forward operator (migration, diffraction summation) of the whole resident cube into
 * image[n_oi][n_ox][n_t] (host).  This is kirchhoffKernel3DWithPadding
 * (src/migration_kernel.cpp:17-383) applied to every output inline of src/main.cpp:257-369. */
int psm_forward(psm_ctx *ctx, float *image);

/* Forward migration from host buffers in one call: traces and vrms [n_il][n_xl][n_t] (host)
 * in, image [n_oi][n_ox][n_t] (host) out.  Pipelined: inline blocks upload on a copy stream,
 * the output inlines whose buffers and Vrms rows are resident migrate (on two alternating
 * compute streams) while later blocks upload, and image rows return on another stream while
 * later output inlines migrate (pinned host buffers let the copies overlap).  Leaves the
 * traces and Vrms resident, as psm_set_traces/_vrms. */
int psm_forward_host(psm_ctx *ctx, const float *traces, const float *vrms, float *image);

/* Same as psm_forward, leaving the image in device memory owned by ctx (enqueued on the ctx
 * stream). */
int psm_forward_async(psm_ctx *ctx);
int psm_synchronize(psm_ctx *ctx);
/* Device pointer of the ctx-owned image [n_oi][n_ox][n_t] (valid until the next
 * psm_set_geometry / psm_destroy). */
int psm_image_device(psm_ctx *ctx, float **dev_image);
/* Copy the ctx-owned image to the host. */
int psm_get_image(psm_ctx *ctx, float *image);
/* Raw CUDA stream of the ctx (a cudaStream_t). */
int psm_stream(psm_ctx *ctx, void **stream);

/* ---- Slabs of output inlines: out-of-core streaming and sharding across GPUs.  No
 * counterpart in the reference, which re-reads each output inline's input window from the
 * file (prepareInputBufferWithPadding, src/migration_kernel.cpp:385-468).  A slab is output
 * inlines [o0, o1) and the input inlines [i0, i1) their buffers read (each output inline o
 * reads [c - m_il - pad_il, c + m_il + 1 + pad_il) around its centre c, clamped to the cube,
 * migration_kernel.cpp:404-409); migrating the slab on its own gives exactly those rows of the
 * whole image. */
typedef struct {
    int32_t o0, o1; /* output inlines */
    int32_t i0, i1; /* input inlines */
} psm_slab;

/* Device bytes a slab of n_in input inlines and n_out output inlines holds while it is
 * migrated (traces as uploaded and in the storage the kernel stages, Vrms, image). */
int64_t psm_slab_bytes(const psm_geom *g, int32_t n_in, int32_t n_out);
/* Split the output inlines into consecutive slabs of at most max_device_bytes each
 * (max_device_bytes <= 0: one slab).  slabs[max_slabs]; *n_slabs the count.
 * PSM_ERR_UNSUPPORTED when one output inline alone exceeds the budget, PSM_ERR_ARG when
 * max_slabs is too small. */
int psm_plan_slabs(const psm_geom *g, const int32_t *out_center, int64_t max_device_bytes,
                   psm_slab *slabs, int32_t max_slabs, int32_t *n_slabs);
/* Split the output inlines into n_parts consecutive slabs of about equal work, the work of
 * output inline o being weight[o] (NULL: 1 each), for sharding over n_parts GPUs. */
int psm_split_slabs(const psm_geom *g, const int32_t *out_center, const double *weight,
                    int32_t n_parts, psm_slab *slabs);
/* Geometry of a slab on its own: n_il = i1 - i0, n_oi = o1 - o0, and local_center[n_oi] the
 * slab's output centres relative to i0 (for psm_set_geometry with traces and Vrms from input
 * inline i0 on). */
int psm_slab_geometry(const psm_geom *g, const int32_t *out_center, const psm_slab *slab,
                      psm_geom *local, int32_t *local_center);
/* Forward migration of a cube held in host memory, streamed through the ctx in slabs of at
 * most max_device_bytes: traces and vrms [n_il][n_xl][n_t] (host) in, image
 * [n_oi][n_ox][n_t] (host) out.  For cubes larger than the GPU's memory.  The input inlines
 * that consecutive slabs share stay on the device; only the new ones are uploaded.
 * Afterwards the ctx holds the last slab's geometry and no readable traces: call
 * psm_set_geometry before using it again. */
int psm_forward_streamed(psm_ctx *ctx, const psm_geom *g, const int32_t *out_center,
                         const float *traces, const float *vrms, float *image,
                         int64_t max_device_bytes);

/* ---- Vrms assembled on the GPU into the ctx's Vrms cube [n_il][n_xl][n_t] (what
 * psm_set_vrms uploads), at sample times t * dt_seconds.  No counterpart in the reference,
 * whose providers loop on the CPU (src/velocity_reader.cpp); the operations and their order
 * are the host providers' (include/psm_host.h), so the cube is the same bit for bit.
 *   psm_set_vrms_table: the text-table provider (:264-370): points (il, xl, time in s, v);
 *     every point blends into every sample with weight 1 / (1 + dist), an exact hit returns its
 *     v, a non-positive result the smallest v.
 *   psm_set_vrms_grid: the SEG-Y provider (:33-261) on its dense grid [g_nil][g_nxl][g_nt]
 *     (sorted labels, missing traces zero, sample interval g_dt): points on grid labels copy
 *     or interpolate their trace in time, others blend the 2x2 label neighbours.
 * il_labels[n_il], xl_labels[n_xl] are the cube's labels. */
int psm_set_vrms_table(psm_ctx *ctx, const int32_t *p_il, const int32_t *p_xl,
                       const double *p_time, const float *p_v, int32_t n_points,
                       const int32_t *il_labels, const int32_t *xl_labels);
int psm_set_vrms_grid(psm_ctx *ctx, const float *grid, const int32_t *g_il, int32_t g_nil,
                      const int32_t *g_xl, int32_t g_nxl, int32_t g_nt, double g_dt,
                      const int32_t *il_labels, const int32_t *xl_labels);
/* The ctx's Vrms cube (host out). */
int psm_get_vrms(psm_ctx *ctx, float *vrms);

/* ---- SEG-Y trace codec on the GPU.  No counterpart in the reference, which decodes and
 * encodes every trace on the CPU (readTraceData, src/segy_utils.cpp:272-318, with ibmToIeee
 * :243-254; writeTrace :598-648 with ieeeToIbm :257-270); the bytes are the same.
 *
 * psm_set_traces_segy uploads n_records trace records exactly as they follow the file's 3600
 * header bytes (a 240-byte header and n_t big-endian samples each; format 1 IBM, anything
 * else IEEE) and decodes them on the GPU into the resident cube: record r fills cube trace
 * position[r] (il_index * n_xl + xl_index), or nothing when position[r] is -1 (zero labels,
 * or a duplicate (IL, XL) that a later record overrides, segy_utils.cpp:164-204).  Traces no
 * record fills are zero.  The upload runs in 32 MB chunks on a second stream, overlapped with
 * the decode when the records are in pinned memory.  The records stay on the device as the
 * header sources of psm_get_image_segy. */
int psm_set_traces_segy(psm_ctx *ctx, const void *records, int64_t n_records, int32_t format,
                        const int32_t *position);
/* Encodes the ctx image as n_oi * n_ox output records (240 + 4 n_t bytes each, host `out`):
 * output trace r = o * n_ox + x copies the header of uploaded record source[r], or, for
 * source[r] = -1, gets a zero header with INLINE_3D@188 = il_label[o] and CROSSLINE_3D@192 =
 * xl_label[x] (segy_utils.cpp:605-620, main.cpp:393-413); samples big-endian, format 1 IBM
 * (the reference's truncating ieeeToIbm; +-inf -> sign|0x7FFFFFFF, NaN -> 0x40000000, where
 * the reference never terminates) or IEEE. */
int psm_get_image_segy(psm_ctx *ctx, void *out, int32_t format, const int32_t *source,
                       const int32_t *il_label, const int32_t *xl_label);
/* The resident fp32 cube [n_il][n_xl][n_t] as uploaded or decoded (host out). */
int psm_get_traces(psm_ctx *ctx, float *data);
/* Overwrite the ctx image [n_oi][n_ox][n_t] from the host (e.g. to encode a given image). */
int psm_set_image(psm_ctx *ctx, const float *image);

/* Adjoint of psm_forward (demigration / spray, M^T): data[n_il][n_xl][n_t] (host, output)
 * from image[n_oi][n_ox][n_t] (host).  Every term of the forward is spread back with its
 * transposed interpolation weights (1 - frac, frac) and the same amplitude weight, so
 * <M d, m> = <d, M^T m> to FP32 summation noise.  Needs geometry and vrms; replaces the
 * resident traces with nothing (they stay). */
int psm_adjoint(psm_ctx *ctx, const float *image, float *data);

/* psm_adjoint on device memory, enqueued on the ctx stream: M^T of the ctx image
 * (psm_image_device; after psm_set_image or a forward) into the ctx's fp32 trace cube, which
 * psm_get_traces then reads.  Before the next forward, upload traces again. */
int psm_adjoint_async(psm_ctx *ctx);

/* The operator pair on caller device memory, enqueued on the ctx stream (psm_stream), with no
 * host copy and no host synchronisation; psm_synchronize waits and reports device errors.
 * For iterative solvers that keep their vectors on the device (least-squares migration
 * sharded over GPUs, where each rank's vectors stay in HBM and only halos cross NVLink).  No
 * counterpart in the reference.
 *   psm_forward_device: image[n_oi][n_ox][n_t] = M data[n_il][n_xl][n_t] (fp32 storage;
 *                       the data become the ctx's resident traces)
 *   psm_adjoint_device: data[n_il][n_xl][n_t] = M^T image[n_oi][n_ox][n_t] (overwritten)
 * Both need geometry and vrms. */
int psm_forward_device(psm_ctx *ctx, const float *d_data, float *d_image);
int psm_adjoint_device(psm_ctx *ctx, const float *d_image, float *d_data);

/* Least-squares migration: `iters` iterations of CG (CGLS) on min ||M^T m - data||^2 from
 * m = 0, with FP32 operators and FP64 inner products and step lengths computed on the GPU.
 * data [n_il][n_xl][n_t] (host) in, image [n_oi][n_ox][n_t] (host) out, resid[iters + 1]
 * (host, may be NULL) the data-residual norms ||M^T m_k - data||.  Overwrites the resident
 * traces. */
int psm_lsm_cg(psm_ctx *ctx, const float *data, float *image, int iters, double *resid);

/* Forward-kernel variants: f32x2-packed or scalar FP32 arithmetic for each pair of 32-sample
 * blocks, 2, 4 or 8 blocks behind one warp-uniform skip test, and 8 or 16 blocks per lane (a
 * tile of 256 or 512 output samples).  All give the same masks and the same terms, bit for
 * bit; they differ in instruction count and shared-memory traffic.  The PAIRS variants (fp32
 * storage) evaluate the travel time once for the two traces at inlines c - d and c + d of one
 * crossline, which share it, and add their two samples before the weight: the same terms,
 * summed in another order (equal to FP32 rounding).  PSM_FWD_DEFAULT lets the
 * library pick (the result of psm_autotune once it has run on the ctx). */
typedef enum {
    PSM_FWD_DEFAULT = 0,
    PSM_FWD_SCALAR_G2 = 1,
    PSM_FWD_SCALAR_G4 = 2,
    PSM_FWD_PACKED_G2 = 3,
    PSM_FWD_PACKED_G4 = 4,
    PSM_FWD_PACKED_G4_J16 = 5,
    PSM_FWD_SCALAR_G4_J16 = 6,
    PSM_FWD_PACKED_G8 = 7,
    PSM_FWD_SCALAR_G8 = 8,
    PSM_FWD_PACKED_G4_O3 = 9,  /* 3 CTAs per SM: 72 registers, 32 KB stages */
    PSM_FWD_SCALAR_G4_O3 = 10,
    PSM_FWD_PAIRS_O3 = 11, /* mirrored inlines c - d, c + d staged as pairs, 3 CTAs per SM */
    PSM_FWD_PAIRS = 12,
    PSM_FWD_PAIRS_J4_O4 = 13, /* pairs, tiles of 128 samples, 4 CTAs per SM (56 registers) */
    PSM_FWD_N_VARIANTS = 14
} psm_fwd_variant;
int psm_set_variant(psm_ctx *ctx, int variant);
int psm_get_variant(psm_ctx *ctx, int *variant);
/* Time one forward launch of every variant on the resident cube (CUDA events on the ctx
 * stream), keep the fastest for this ctx.  ms[PSM_FWD_N_VARIANTS] (may be NULL) receives the
 * times, ms[0] unused; *best (may be NULL) the chosen variant. */
int psm_autotune(psm_ctx *ctx, float *ms, int *best);

/* Number of (output sample, input trace) terms that pass every mask of the reference
 * (migration_kernel.cpp:166, :207/:286, :226/:298) over the real input traces, counted on
 * the GPU with the forward kernel's own arithmetic. */
int psm_count_terms(psm_ctx *ctx, int64_t *n_terms);
/* The same count per output inline: per_row[n_oi]. */
int psm_count_terms_rows(psm_ctx *ctx, int64_t *per_row);

/* ---- Batched migration: several problems (velocity-scan panels over one cube, uneven
 * sub-volumes with their own Vrms) in ONE persistent launch, replayed as a CUDA graph.  No
 * counterpart in the reference, which migrates one cube with one velocity field per run
 * (src/main.cpp:291-361); each problem is exactly that run's operator. */
typedef enum {
    PSM_VRMS_CUBE = 0,     /* vrms [n_il][n_xl][n_t], as psm_set_vrms */
    PSM_VRMS_TRACE = 1,    /* vrms [n_t]: one Vrms(t) for every output point */
    PSM_VRMS_CONSTANT = 2  /* velocity for every point and sample (a scan panel) */
} psm_vrms_kind;

typedef struct {
    psm_geom geom;             /* amp_correction, precision and compensated equal for all */
    const int32_t *out_center; /* [geom.n_oi] or NULL, as psm_set_geometry */
    const float *traces;       /* host [n_il][n_xl][n_t]; problems that pass the same pointer
                                  and grid share one device copy */
    const float *vrms;         /* see vrms_kind; unused for PSM_VRMS_CONSTANT */
    int32_t vrms_kind;
    float velocity;            /* PSM_VRMS_CONSTANT */
} psm_problem;

typedef struct psm_batch psm_batch;

typedef enum {
    PSM_BATCH_PERSISTENT = 0,  /* one persistent launch over every problem's tiles */
    PSM_BATCH_PER_PROBLEM = 1, /* one grid launch per problem */
    PSM_BATCH_ONE_GRID = 2     /* one grid launch over every problem's tiles, a CTA per tile in
                                  the tile order (the block scheduler balances the load) */
} psm_batch_mode;

/* At most 184 problems (PSM_ERR_UNSUPPORTED beyond): their parameters travel as one kernel
 * argument.  Uploads every problem (the host arrays are read again by psm_batch_reload, so
 * they must stay valid while the batch lives) and builds the tile lists (psm_tile_order).
 * Images stay on the device. */
int psm_batch_create(psm_ctx *ctx, const psm_problem *problems, int n_problems,
                     psm_batch **out);
int psm_batch_destroy(psm_batch *batch);
int psm_batch_reload(psm_batch *batch); /* re-upload traces and Vrms from the host arrays */
/* Either mode runs as one CUDA graph (captured on the first run of a variant / order /
 * mode, then replayed). */
int psm_batch_set_mode(psm_batch *batch, int mode);
int psm_batch_get_mode(psm_batch *batch, int *mode);
int psm_batch_set_variant(psm_batch *batch, int variant);
int psm_batch_get_variant(psm_batch *batch, int *variant);

/* Order in which the persistent CTAs take the tiles. */
typedef enum {
    PSM_ORDER_DEPTH_FIRST = 0, /* deepest time tiles first, problems interleaved per tile */
    PSM_ORDER_PROBLEM = 1      /* problem after problem, each in grid order */
} psm_tile_order;
int psm_batch_set_order(psm_batch *batch, int order);
int psm_batch_get_order(psm_batch *batch, int *order);
/* Times one run per distinct kernel variant on each of five schedules (0 persistent
 * depth-first, 1 persistent problem order, 2 one launch per problem, 3 one grid depth-first,
 * 4 one grid problem order) and keeps the fastest
 * variant, order and mode; ms[5 * PSM_FWD_N_VARIANTS] (may be NULL) receives the times at
 * [schedule * PSM_FWD_N_VARIANTS + variant], 0 for variants not run. */
int psm_batch_autotune(psm_batch *batch, float *ms, int *best, int *best_order,
                       int *best_mode);
int psm_batch_run_async(psm_batch *batch); /* on the context's stream */
int psm_batch_synchronize(psm_batch *batch);
int psm_batch_run(psm_batch *batch);       /* run_async + synchronize */
int psm_batch_image_device(psm_batch *batch, int problem, float **dev_image);
int psm_batch_get_image(psm_batch *batch, int problem, float *image);
/* Terms over all problems (psm_count_terms of each). */
int psm_batch_count_terms(psm_batch *batch, int64_t *n_terms);

/* Per-inline drop-in for MigrationKernel::kirchhoffKernel3DWithPadding
 * (include/migration_kernel.h:16-31, src/migration_kernel.cpp:17-383): the same arguments,
 * output_slice flat [n_out_xl][n_t] instead of vector<vector<float>>; xl_pos_indices is
 * unused (as in the reference) and may be NULL.  Uploads the buffer on each call, so it is
 * the slow path; the resident-cube calls above are the fast path.  Thread-safe: each host
 * thread gets its own device staging. */
int psm_kirchhoff_inline(const float *input_buffer, size_t n_buf_il, size_t n_buf_xl,
                         size_t n_t, const float *velocity_slice, float *output_slice,
                         size_t n_out_xl, const int32_t *il_pos_indices,
                         const int32_t *xl_pos_indices, int32_t current_il_pos,
                         int32_t current_xl_start, float dt, const float *t0_times,
                         float tan_theta_sq, float inline_bin_size,
                         float crossline_bin_size, int amp_correction);
/* Message of the last psm_kirchhoff_inline failure on this thread. */
const char *psm_kirchhoff_inline_error(void);

/* ---- Measured throughput of the SM limbs the summation draws on (no counterpart in the
 * reference; a measurement for the roofline).  Probe kernels run independent operations on
 * every SM at once; each rate is operations per SM clock per SM (from clock64 spans, so it
 * does not depend on the clock the GPU ran at), and sm_clock_mhz the clock those spans imply
 * over the CUDA-event time.  The "slope" rates put lane l of a warp at element floor(4 l / 5),
 * the pattern of 32 consecutive output samples on one trace (ds/dt0 = t0 / t, about 0.8). */
typedef struct {
    double sm_clock_mhz;
    int32_t n_sm;
    double rsqrt_per_clk_sm;             /* MUFU rsqrt results */
    double ffma_per_clk_sm;              /* scalar fp32 FMAs */
    double ffma2_per_clk_sm;             /* fp32 FMAs issued as fma.rn.f32x2 (2 per lane) */
    double lds64_bytes_per_clk_sm;       /* 8-byte shared loads, consecutive lanes */
    double lds64_slope_bytes_per_clk_sm; /* 8-byte shared loads, slope pattern */
    double atom_per_clk_sm;              /* shared fp32 atomicAdd, consecutive lanes */
    double atom_slope_per_clk_sm;        /* the same, slope pattern */
    double red_per_clk_sm;               /* red.shared.add.f32 (no return), consecutive */
    double red_slope_per_clk_sm;         /* the same, slope pattern */
    double atom_u32_per_clk_sm;          /* shared 32-bit integer atomicAdd, consecutive */
    double atom_u32_slope_per_clk_sm;    /* the same, slope pattern */
    double atom_u64_per_clk_sm;          /* shared 64-bit integer atomicAdd, consecutive */
    double atom_u64_slope_per_clk_sm;    /* the same, slope pattern */
} psm_limbs;
int psm_measure_limbs(int device, psm_limbs *out);

/* Forward migration that allocates no device memory (this entry point has no counterpart in
 * the reference).  It is for callers that must not call cudaMalloc: applications whose device
 * memory is owned by their own pool or framework allocator, and pipelines that set up all
 * memory once and cannot afford the implicit device synchronisation of cudaMalloc/cudaFree.
 * The caller owns every input and output; all are device pointers:
 *   d_pairs   [n_il][n_xl][ns] pairs of floats (d[t], d[t+1] - d[t]), ns = (n_t + 7) & ~7,
 *             d beyond n_t - 1 taken as 0; 16-byte aligned
 *   d_vrms    [n_il][n_xl][n_t] Vrms of the output points
 *   d_image   [n_oi][n_ox][n_t] output, fully overwritten
 * g and out_center (host, [n_oi] or NULL) mean what they mean for psm_set_geometry; stream is
 * a cudaStream_t (NULL: the default stream).  The call returns when the image is complete.
 * Its only working memory is one file-scope device array of PSM_NOALLOC_SCRATCH_BYTES
 * (192 KiB), which every GPU that loads the library holds until the process exits; it limits
 * n_oi <= 4096, n_il <= 4096 and n_t <= 16384 (PSM_ERR_UNSUPPORTED beyond).  The first call on
 * a device looks up that array's device address, so make it before any stream capture.  All
 * calls share the array and it keeps the last call's contents: calls that overlap on the GPU
 * race, so serialise them. */
#define PSM_NOALLOC_SCRATCH_BYTES (192 * 1024)
int psm_forward_noalloc(const psm_geom *g, const int32_t *out_center, const float *d_pairs,
                        const float *d_vrms, float *d_image, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* PSM_H */
