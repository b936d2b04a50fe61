/* CPU check of the forward kernel's per-sample pass bound search (pass_bound in
 * poststackmig3d_b200/csrc/psm_kernels.cuh), built and run by tests/test_pass_bound_cpu.py.
 *
 * A term passes the reference's range mask when floor(fl(sqrt(fma(f4, r2, t0^2))) * inv_dt)
 * < n_t - 1 (src/migration_kernel.cpp:209-226), in IEEE FP32.  The test is monotone in r2,
 * so the largest passing r2 in [0, md2] is one float bit pattern, which a bisection of all of
 * [0, md2] finds.  The kernel instead starts from an estimate of the boundary and gallops
 * outwards to a bracket before it bisects.  This program restates both searches with the same
 * FP32 operations (compile with -ffp-contract=off) and checks, over seeded (v, t0, dt, n_t,
 * aperture) cases, that the galloping search returns the bisection's bound from the kernel's
 * estimate, from a perturbed estimate and from a random start, and counts the evaluations.
 * Prints one line: cases, cases that needed a search, mismatches, evaluations per search. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static unsigned bits_of(float f) { unsigned u; memcpy(&u, &f, 4); return u; }
static float float_of(unsigned u) { float f; memcpy(&f, &u, 4); return f; }

static long n_eval;

/* the reference's range test for one r2 */
static int range_ok(float r2, float f4, float t0sq, float inv_dt, float ntm1f) {
    ++n_eval;
    volatile float x = fmaf(f4, r2, t0sq);
    volatile float s = sqrtf(x);
    volatile float m = s * inv_dt;
    return m < ntm1f;
}

typedef struct { int valid; float t0sq, f4, md2; } point;

/* per-sample constants in the reference's operation order (migration_kernel.cpp:115-144) */
static point point_of(float v, float t0, float tan2) {
    point p;
    p.valid = v >= 1e-5f && t0 >= 1e-5f;
    volatile float a = t0 * t0; p.t0sq = a;
    volatile float d = fmaf(v, v, 1e-10f);
    volatile float iv = 1.0f / d;
    volatile float f4 = 4.0f * iv; p.f4 = f4;
    volatile float vt = v * t0; vt = vt * 0.5f;
    volatile float md = vt * vt; md = md * tan2; p.md2 = md;
    return p;
}

/* start: 0 plain bisection; 1 the kernel's estimate; 2 the estimate times 1.01; 3 random */
static float bound(point p, float inv_dt, float ntm1f, int start) {
    if (!p.valid || !(p.md2 >= 0.0f)) return -1.0f;
    if (range_ok(p.md2, p.f4, p.t0sq, inv_dt, ntm1f)) return p.md2;
    if (!range_ok(0.0f, p.f4, p.t0sq, inv_dt, ntm1f)) return -1.0f;
    unsigned lo = 0u, hi = bits_of(p.md2);  /* passes at lo, fails at hi */
    if (start && hi - lo > 1u) {
        volatile float a = ntm1f / inv_dt;
        volatile float num = fmaf(a, a, -p.t0sq);
        volatile float e = num / p.f4;
        if (start == 2) e = e * 1.01f;
        unsigned m = e > 0.0f ? bits_of(e) : 0u;
        if (start == 3) m = (unsigned)rand() * 2654435761u;
        if (m < lo + 1u) m = lo + 1u;
        if (m > hi - 1u) m = hi - 1u;
        unsigned step = 1u;
        if (range_ok(float_of(m), p.f4, p.t0sq, inv_dt, ntm1f)) {
            lo = m;
            while (hi - lo > step) {
                unsigned c = lo + step;
                if (!range_ok(float_of(c), p.f4, p.t0sq, inv_dt, ntm1f)) { hi = c; break; }
                lo = c;
                step <<= 1;
            }
        } else {
            hi = m;
            while (hi - lo > step) {
                unsigned c = hi - step;
                if (range_ok(float_of(c), p.f4, p.t0sq, inv_dt, ntm1f)) { lo = c; break; }
                hi = c;
                step <<= 1;
            }
        }
    }
    while (hi - lo > 1u) {
        unsigned mid = lo + ((hi - lo) >> 1);
        if (range_ok(float_of(mid), p.f4, p.t0sq, inv_dt, ntm1f)) lo = mid; else hi = mid;
    }
    return float_of(lo);
}

int main(void) {
    const float dts[] = {0.001f, 0.002f, 0.004f};
    const int nts[] = {101, 501, 751, 1001, 2001};
    const float tan2s[] = {0.0f, 0.0717967f, 0.3333333f, 1.0f, 3.0f, 1e4f};
    long cases = 0, searched = 0, bad = 0, ev_bisect = 0, ev_gallop = 0;
    srand(7);
    for (int id = 0; id < 3; ++id)
        for (int in = 0; in < 5; ++in)
            for (int ia = 0; ia < 6; ++ia) {
                const float dt = dts[id], inv_dt = 1.0f / dt, ntm1f = (float)(nts[in] - 1);
                for (int k = 0; k < 4000; ++k) {
                    const float t0 = (float)((double)(rand() % nts[in]) * dt);
                    float v;
                    switch (rand() % 5) {  /* velocities from field values to degenerate */
                        case 0: v = 1500.0f + 3000.0f * (rand() / (float)RAND_MAX); break;
                        case 1: v = (float)(rand() % 10000); break;
                        case 2: v = 1e-5f * (float)(1 + rand() % 100); break;
                        case 3: v = 1e-3f * (float)(rand() % 1000); break;
                        default: v = float_of(bits_of(1500.0f) + (unsigned)(rand() % 100000) - 50000u);
                    }
                    const point p = point_of(v, t0, tan2s[ia]);
                    n_eval = 0;
                    const float b0 = bound(p, inv_dt, ntm1f, 0);
                    const long e0 = n_eval;
                    n_eval = 0;
                    const float b1 = bound(p, inv_dt, ntm1f, 1);
                    const long e1 = n_eval;
                    const float b2 = bound(p, inv_dt, ntm1f, 2);
                    const float b3 = bound(p, inv_dt, ntm1f, 3);
                    ++cases;
                    if (e0 > 2) { ++searched; ev_bisect += e0; ev_gallop += e1; }
                    if (bits_of(b1) != bits_of(b0) || bits_of(b2) != bits_of(b0) ||
                        bits_of(b3) != bits_of(b0))
                        ++bad;
                }
            }
    printf("cases %ld searched %ld mismatches %ld bisection %.2f gallop %.2f\n", cases,
           searched, bad, (double)ev_bisect / (double)(searched ? searched : 1),
           (double)ev_gallop / (double)(searched ? searched : 1));
    return bad != 0;
}
