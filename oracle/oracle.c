/* TEST INFRASTRUCTURE ONLY -- CPU checker for the Kirchhoff summation path.  See oracle.h.
 *
 * Every function below restates sergeevsn/poststackmig3d's src/migration_kernel.cpp
 * (line numbers cited inline).  Compiled by oracle/Makefile with -ffp-contract=off and no
 * fast-math, so each C expression rounds exactly where it is written; ORACLE_CONTRACT
 * switches the three multiply-add sites to fmaf() to model the reference's GCC build.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Per output sample constants, migration_kernel.cpp:115-144. */
typedef struct {
    int valid;
    float t0sq, v, f4, maxd2;
    int xs, xe; /* crossline window [xs, xe) in buffer coordinates */
} point_t;

static point_t point_setup(float t0v, float v, float tan2, float inv_dxl, int64_t xb,
                           int64_t n_buf_xl, int contract) {
    point_t p;
    memset(&p, 0, sizeof p);
    if (!(v >= 1e-5f && t0v >= 1e-5f)) return p; /* :121 */
    p.valid = 1;
    p.t0sq = t0v * t0v;                           /* :125 */
    p.v = v;
    float vsq = v * v;                            /* :127 */
    /* :128; the reference's build fuses v*v + 1e-10 */
    float inv_vsq = 1.0f / (contract ? fmaf(v, v, 1e-10f) : vsq + 1e-10f);
    p.f4 = 4.0f * inv_vsq;                        /* :129 */
    float vth = v * t0v * 0.5f;                   /* :133 */
    p.maxd2 = vth * vth * tan2;                   /* :134 */
    float max_r = sqrtf(p.maxd2);                 /* :137 */
    int mxl = (int)(max_r * inv_dxl) + 1;         /* :138 */
    int64_t xs = xb - mxl, xe = xb + mxl + 1;     /* :141-142 */
    p.xs = (int)(xs < 0 ? 0 : xs);
    p.xe = (int)(xe > n_buf_xl ? n_buf_xl : xe);
    return p;
}

/* One term (migration_kernel.cpp:282-318 scalar path; the AVX path :197-276 evaluates the
 * same expressions lane-wise).  Returns 0 when a mask rejects it.  lo/frac/w describe the
 * FP32 evaluation; *th_out the FP32 travel time. */
typedef struct {
    int lo;
    float frac, th, w;
} term_t;

static int term_eval(const point_t *p, float dx2, int64_t dk, float d_xl, float inv_dt,
                     int64_t n_t, int amp, int contract, term_t *tm) {
    float dy = (float)dk * d_xl;                                  /* :282 */
    float r2 = contract ? fmaf(dy, dy, dx2) : dx2 + dy * dy;      /* :283-284 */
    if (r2 > p->maxd2) return 0;                                  /* :286 */
    float th2 = contract ? fmaf(p->f4, r2, p->t0sq) : p->t0sq + p->f4 * r2;
    float th = sqrtf(th2);                                        /* :291 */
    float s = th * inv_dt;                                        /* :294 */
    int lo = (int)s;                                              /* :295 */
    if (!(lo < (int)n_t - 1)) return 0;                           /* :298 */
    tm->lo = lo;
    tm->frac = s - (float)lo;                                     /* :299 */
    tm->th = th;
    tm->w = 1.0f;
    if (amp) {                                                    /* :312-316 */
        float vsq = p->v * p->v;
        float den = contract ? fmaf(th, vsq, 1e-10f) : th * vsq + 1e-10f;
        tm->w = 1.0f / den;
    }
    (void)r2;
    return 1;
}

/* FP64 values for a term whose masks passed in FP32. */
static void term_f64(const point_t *p, double dx_d, int64_t dk, float d_xl, float dt,
                     float t0v, int64_t n_t, int amp, double *frac_d, int *lo_d,
                     double *w_d) {
    double dy_d = (double)dk * (double)d_xl;
    double vd = (double)p->v;
    double f4 = 4.0 / (vd * vd + 1e-10);
    double th = sqrt((double)t0v * (double)t0v + f4 * (dx_d * dx_d + dy_d * dy_d));
    double s = th / (double)dt;
    double fl = floor(s);
    if (fl > (double)(n_t - 2)) fl = (double)(n_t - 2);
    if (fl < 0.0) fl = 0.0;
    *lo_d = (int)fl;
    *frac_d = s - fl;
    *w_d = amp ? 1.0 / (th * vd * vd + 1e-10) : 1.0;
}

/* Trace source: buffer inline i, buffer crossline b -> data trace or zeros. */
typedef struct {
    const float *data;
    int64_t nxd, xoff, il0, n_t;
} src_t;

static const float *src_trace(const src_t *s, int64_t i, int64_t b) {
    int64_t xc = b - s->xoff;
    if (xc < 0 || xc >= s->nxd) return NULL;
    return s->data + ((s->il0 + i) * s->nxd + xc) * s->n_t;
}

/* One output trace: buffer crossline xb, all t. */
static void trace_forward(const src_t *src, int64_t n_buf_il, int64_t n_buf_xl, int64_t n_t,
                          const float *dx2, const double *dxd, const float *vel_x, int64_t xb,
                          float dt, const float *t0, float tan2, float d_xl, int amp,
                          int flags, float *o32, double *o64, int64_t *cnt_all,
                          int64_t *cnt_real) {
    const int contract = (flags & ORACLE_CONTRACT) != 0;
    const int f64 = (flags & ORACLE_F64) != 0;
    const int avx = (flags & ORACLE_AVX_ORDER) != 0;
    const float inv_dt = 1.0f / dt;             /* :44 */
    const float inv_dxl = 1.0f / d_xl;          /* :45 */
    for (int64_t t = 0; t < n_t; ++t) {
        float v = vel_x ? vel_x[t] : 0.0f;
        point_t p = point_setup(t0[t], v, tan2, inv_dxl, xb, n_buf_xl, contract);
        if (!p.valid) { /* :148-151 */
            if (o32) o32[t] = 0.0f;
            if (o64) o64[t] = 0.0;
            continue;
        }
        float acc = 0.0f;
        double acc_d = 0.0;
        for (int64_t i = 0; i < n_buf_il; ++i) {
            if (dx2[i] > p.maxd2) continue; /* :166 */
            float lane[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            int64_t nsimd = avx ? (p.xe - p.xs) / 8 : 0;
            int64_t kv_end = p.xs + nsimd * 8;
            for (int64_t k = p.xs; k < p.xe; ++k) {
                term_t tm;
                if (!term_eval(&p, dx2[i], k - xb, d_xl, inv_dt, n_t, amp, contract, &tm))
                    continue;
                const float *tr = src_trace(src, i, k);
                ++*cnt_all;
                if (tr) ++*cnt_real;
                if (f64) {
                    if (!tr) continue;
                    double fr, w;
                    int lo;
                    term_f64(&p, dxd[i], k - xb, d_xl, dt, t0[t], n_t, amp, &fr, &lo, &w);
                    double a = tr[lo], b = tr[lo + 1];
                    acc_d += (a + fr * (b - a)) * w;
                } else {
                    float a = tr ? tr[tm.lo] : 0.0f, b = tr ? tr[tm.lo + 1] : 0.0f;
                    float val = fmaf(tm.frac, b - a, a); /* simdInterpolate :544-550 */
                    val = val * tm.w;
                    if (k < kv_end)
                        lane[(k - p.xs) & 7] += val;
                    else
                        acc += val;
                }
            }
            if (avx)
                for (int l = 0; l < 8; ++l) acc += lane[l]; /* :323-327 */
        }
        if (o32) o32[t] = f64 ? (float)acc_d : acc;
        if (o64) o64[t] = f64 ? acc_d : (double)acc;
    }
}

int64_t oracle_kirchhoff_inline(const float *buf, int64_t n_buf_il, int64_t n_buf_xl,
                                int64_t n_t, const float *vel, float *out, double *out64,
                                int64_t n_out_xl, const int32_t *il_pos,
                                int32_t cur_il_pos, int32_t cur_xl_start, float dt,
                                const float *t0, float tan2, float d_il, float d_xl,
                                int amp, int flags) {
    if (n_out_xl == 0 || n_t == 0) return 0; /* :35-37 */
    int32_t cur = (cur_il_pos >= 0 && cur_il_pos < (int32_t)n_buf_il) ? il_pos[cur_il_pos]
                                                                         : 0; /* :48-49 */
    float *dx2 = (float *)malloc(sizeof(float) * (size_t)(n_buf_il ? n_buf_il : 1));
    double *dxd = (double *)malloc(sizeof(double) * (size_t)(n_buf_il ? n_buf_il : 1));
    for (int64_t i = 0; i < n_buf_il; ++i) { /* :51-56 */
        float dx = (float)(il_pos[i] - cur) * d_il;
        dx2[i] = dx * dx;
        dxd[i] = (double)(il_pos[i] - cur) * (double)d_il;
    }
    src_t src = {buf, n_buf_xl, 0, 0, n_t};
    int64_t ca = 0, cr = 0;
    for (int64_t x = 0; x < n_out_xl; ++x) {
        int64_t xb = cur_xl_start + x; /* :77 */
        float *o32 = out ? out + x * n_t : NULL;
        double *o64 = out64 ? out64 + x * n_t : NULL;
        if (xb < 0 || xb >= n_buf_xl) { /* :79-85 */
            for (int64_t t = 0; t < n_t; ++t) {
                if (o32) o32[t] = 0.0f;
                if (o64) o64[t] = 0.0;
            }
            continue;
        }
        trace_forward(&src, n_buf_il, n_buf_xl, n_t, dx2, dxd, vel + xb * n_t, xb, dt, t0,
                      tan2, d_xl, amp, flags, o32, o64, &ca, &cr);
    }
    free(dx2);
    free(dxd);
    return ca;
}

/* Buffer geometry of one output inline (migration_kernel.cpp:404-416). */
static void buffer_range(int32_t c, int32_t n_il, int32_t m_il, int32_t pad_il,
                         int32_t *il0, int32_t *il1) {
    int32_t rs = c - m_il < 0 ? 0 : c - m_il;
    int32_t re = c + m_il + 1 > n_il ? n_il : c + m_il + 1;
    *il0 = rs - pad_il < 0 ? 0 : rs - pad_il;
    *il1 = re + pad_il > n_il ? n_il : re + pad_il;
}

void oracle_migrate_volume(const float *data, const float *vrms, int32_t n_il, int32_t n_xl,
                           int32_t n_t, const int32_t *out_center, int32_t n_oi,
                           int32_t n_ox, int32_t pad_il, int32_t pad_xl, int32_t m_il,
                           float dt, const float *t0, float tan2, float d_il, float d_xl,
                           int amp, int flags, int n_threads, float *out, double *out64,
                           int64_t *counts) {
    const int64_t n_buf_xl = (int64_t)n_xl + 2 * (int64_t)pad_xl;
    int64_t ca = 0, cr = 0;
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#else
    (void)n_threads;
#endif
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : ca, cr)
    for (int64_t ox = 0; ox < (int64_t)n_oi * n_ox; ++ox) {
        int32_t o = (int32_t)(ox / n_ox);
        int64_t x = ox % n_ox;
        int32_t c = out_center[o];
        int32_t il0, il1;
        buffer_range(c, n_il, m_il, pad_il, &il0, &il1);
        int64_t nb = il1 - il0;
        float dx2[nb > 0 ? nb : 1];
        double dxd[nb > 0 ? nb : 1];
        for (int64_t i = 0; i < nb; ++i) {
            float dx = (float)((il0 + (int32_t)i) - c) * d_il;
            dx2[i] = dx * dx;
            dxd[i] = (double)((il0 + (int32_t)i) - c) * (double)d_il;
        }
        float *o32 = out ? out + ((int64_t)o * n_ox + x) * n_t : NULL;
        double *o64 = out64 ? out64 + ((int64_t)o * n_ox + x) * n_t : NULL;
        int64_t xb = x; /* current_xl_start = 0 (main.cpp:362) */
        int64_t xc = xb - pad_xl;
        const float *vel_x = (xc >= 0 && xc < n_xl && xb < n_buf_xl)
                                 ? vrms + ((int64_t)c * n_xl + xc) * n_t
                                 : NULL; /* migration_kernel.cpp:486-510: padding v = 0 */
        if (xb >= n_buf_xl) {
            for (int64_t t = 0; t < n_t; ++t) {
                if (o32) o32[t] = 0.0f;
                if (o64) o64[t] = 0.0;
            }
            continue;
        }
        src_t src = {data, n_xl, pad_xl, il0, n_t};
        int64_t a = 0, r = 0;
        trace_forward(&src, nb, n_buf_xl, n_t, dx2, dxd, vel_x, xb, dt, t0, tan2, d_xl, amp,
                      flags, o32, o64, &a, &r);
        ca += a;
        cr += r;
    }
    if (counts) {
        counts[0] = ca;
        counts[1] = cr;
    }
}

/* Terms per output row r in [r0, r1) without summing: for each output sample and buffer
 * inline the passing crosslines are |k - x| <= d (both masks grow with r^2), d found by a
 * square-root guess and exact-mask fix-ups.  Real input traces only. */
void oracle_count_rows(const float *vrms, int32_t n_il, int32_t n_xl, int32_t n_t,
                       const int32_t *out_center, int32_t r0, int32_t r1, int32_t n_ox,
                       int32_t pad_il, int32_t pad_xl, int32_t m_il, float dt,
                       const float *t0, float tan2, float d_il, float d_xl, int amp,
                       int flags, int n_threads, int64_t *rows_out) {
    const int contract = (flags & ORACLE_CONTRACT) != 0;
    const int64_t n_buf_xl = (int64_t)n_xl + 2 * (int64_t)pad_xl;
    const float inv_dt = 1.0f / dt;
    const float inv_dxl = 1.0f / d_xl;
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#else
    (void)n_threads;
#endif
    for (int32_t r = r0; r < r1; ++r) {
        int32_t c = out_center[r];
        int32_t il0, il1;
        buffer_range(c, n_il, m_il, pad_il, &il0, &il1);
        int64_t total = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : total)
        for (int64_t xb = 0; xb < n_ox; ++xb) {
            int64_t xc = xb - pad_xl;
            if (xb >= n_buf_xl || xc < 0 || xc >= n_xl) continue;
            const float *vel_x = vrms + ((int64_t)c * n_xl + xc) * n_t;
            for (int64_t t = 0; t < n_t; ++t) {
                point_t p = point_setup(t0[t], vel_x[t], tan2, inv_dxl, xb, n_buf_xl, contract);
                if (!p.valid) continue;
                for (int32_t il = il0; il < il1; ++il) {
                    float dx = (float)(il - c) * d_il;
                    float dx2 = dx * dx;
                    if (dx2 > p.maxd2) continue;
                    term_t tm;
                    if (!term_eval(&p, dx2, 0, d_xl, inv_dt, n_t, amp, contract, &tm))
                        continue;
                    float rem = p.maxd2 - dx2;
                    int64_t d = (int64_t)(sqrtf(rem > 0.0f ? rem : 0.0f) * inv_dxl);
                    if (d > n_buf_xl) d = n_buf_xl;
                    while (d > 0 &&
                           !term_eval(&p, dx2, d, d_xl, inv_dt, n_t, amp, contract, &tm))
                        --d;
                    while (d < n_buf_xl &&
                           term_eval(&p, dx2, d + 1, d_xl, inv_dt, n_t, amp, contract, &tm))
                        ++d;
                    /* real crosslines within the reference's window [xs, xe) */
                    int64_t lo = xb - d, hi = xb + d;
                    if (lo < p.xs) lo = p.xs;
                    if (hi > p.xe - 1) hi = p.xe - 1;
                    if (lo < pad_xl) lo = pad_xl;
                    if (hi > pad_xl + n_xl - 1) hi = pad_xl + n_xl - 1;
                    if (hi >= lo) total += hi - lo + 1;
                }
            }
        }
        rows_out[r - r0] = total;
    }
}

void oracle_adjoint_volume(const double *image, const float *vrms, int32_t n_il,
                           int32_t n_xl, int32_t n_t, const int32_t *out_center,
                           int32_t n_oi, int32_t n_ox, int32_t pad_il, int32_t pad_xl,
                           int32_t m_il, float dt, const float *t0, float tan2, float d_il,
                           float d_xl, int amp, int flags, int n_threads, double *data_out) {
    const int contract = (flags & ORACLE_CONTRACT) != 0;
    const int64_t n_buf_xl = (int64_t)n_xl + 2 * (int64_t)pad_xl;
    const float inv_dt = 1.0f / dt;
    const float inv_dxl = 1.0f / d_xl;
    memset(data_out, 0, sizeof(double) * (size_t)n_il * n_xl * n_t);
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#else
    (void)n_threads;
#endif
    /* One data inline il per iteration: it receives the terms of every output inline whose
     * buffer holds it, in (o, xb, t, k) order -- the order of the serial loop nest over o, xb,
     * t, il, k -- so the sums do not depend on the thread count. */
#pragma omp parallel for schedule(dynamic, 1)
    for (int32_t il = 0; il < n_il; ++il) {
        for (int32_t o = 0; o < n_oi; ++o) {
            int32_t c = out_center[o];
            int32_t il0, il1;
            buffer_range(c, n_il, m_il, pad_il, &il0, &il1);
            if (il < il0 || il >= il1) continue;
            float dx = (float)(il - c) * d_il;
            float dx2 = dx * dx;
            double dxd = (double)(il - c) * (double)d_il;
            for (int64_t xb = 0; xb < n_ox && xb < n_buf_xl; ++xb) {
                int64_t xc = xb - pad_xl;
                if (xc < 0 || xc >= n_xl) continue; /* v = 0 there: no terms */
                const float *vel_x = vrms + ((int64_t)c * n_xl + xc) * n_t;
                for (int64_t t = 0; t < n_t; ++t) {
                    double m = image[((int64_t)o * n_ox + xb) * n_t + t];
                    if (m == 0.0) continue;
                    point_t p = point_setup(t0[t], vel_x[t], tan2, inv_dxl, xb, n_buf_xl,
                                            contract);
                    if (!p.valid) continue;
                    if (dx2 > p.maxd2) continue;
                    for (int64_t k = p.xs; k < p.xe; ++k) {
                        int64_t kc = k - pad_xl;
                        if (kc < 0 || kc >= n_xl) continue;
                        term_t tm;
                        if (!term_eval(&p, dx2, k - xb, d_xl, inv_dt, n_t, amp, contract,
                                       &tm))
                            continue;
                        double *dtr = data_out + ((int64_t)il * n_xl + kc) * n_t;
                        if (flags & ORACLE_F64) {
                            double fr, w;
                            int lo;
                            term_f64(&p, dxd, k - xb, d_xl, dt, t0[t], n_t, amp, &fr, &lo,
                                     &w);
                            dtr[lo] += (1.0 - fr) * w * m;
                            dtr[lo + 1] += fr * w * m;
                        } else {
                            dtr[tm.lo] += (1.0 - (double)tm.frac) * (double)tm.w * m;
                            dtr[tm.lo + 1] += (double)tm.frac * (double)tm.w * m;
                        }
                    }
                }
            }
        }
    }
}
