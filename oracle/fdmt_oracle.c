/* ORACLE — test infrastructure only (see oracle.h).
 *
 * Restatement of the reference's Keith-style FDMT, single threaded:
 *   plan      MyVSLib_C++/FDMT/FdmtB.cpp:201-204 (calc_deltaT), :206-227
 *             (calcNextStateConfig), :238-245 (calcCumSum_),
 *             MyVSLib_C++/FDMT/FdmtCpu.cpp:143-194 (create_config)
 *   level 0   MyVSLib_C++/FDMT/FdmtCpu.cpp:314-367 (fnc_initC)
 *   level i   MyVSLib_C++/FDMT/FdmtCpu.cpp:252-311 (fncFdmtIterationC)
 *   driver    MyVSLib_C++/FDMT/FdmtCpu.cpp:197-249 (process_image)
 * Float expressions keep the reference's types and evaluation order (float
 * products squared before the double reciprocal, float coefficients, float
 * row index products truncated to int), so with -ffp-contract=off the FP32
 * result is bit-identical to CFdmtCpu run on one thread.
 */
#include "oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_MAXL 40

typedef struct {
    float fmin, fmax;
    int nchan, max_dt, niter;
    int nsub[ORC_MAXL];
    int* rows[ORC_MAXL]; /* rows per sub-band */
    int* cum[ORC_MAXL];  /* nsub+1 cumulative rows */
    float* freq[ORC_MAXL];
} oplan;

static int delta_t(const oplan* p, float f0, float f1) {
    float f0sq = f0 * f0, f1sq = f1 * f1;
    float lo = p->fmin * p->fmin, hi = p->fmax * p->fmax;
    double num = 1.0 / (double)f0sq - 1.0 / (double)f1sq;
    double den = 1.0 / (double)lo - 1.0 / (double)hi;
    return (int)ceil(num / den * ((double)p->max_dt - 1.0));
}

static float band_delay(float flo, float fhi) {
    float a = flo * flo, b = fhi * fhi;
    return (float)(1.0 / (double)a - 1.0 / (double)b);
}

int orc_fdmt_niter(int nchan) {
    int q = nchan, n = 0;
    while (q > 1) { q = (q & 1) ? q / 2 + 1 : q / 2; ++n; }
    return n;
}

static void plan_free(oplan* p) {
    for (int l = 0; l <= p->niter && l < ORC_MAXL; ++l) {
        free(p->rows[l]); free(p->cum[l]); free(p->freq[l]);
    }
}

static int plan_build(oplan* p, float fmin, float fmax, int nchan, int max_dt) {
    memset(p, 0, sizeof(*p));
    if (nchan < 2 || max_dt < 1 || !(fmax > fmin)) return -1;
    p->fmin = fmin; p->fmax = fmax; p->nchan = nchan; p->max_dt = max_dt;
    p->niter = orc_fdmt_niter(nchan);
    if (p->niter + 1 > ORC_MAXL) return -1;
    for (int l = 0; l <= p->niter; ++l) {
        p->rows[l] = (int*)calloc((size_t)nchan + 1, sizeof(int));
        p->cum[l] = (int*)calloc((size_t)nchan + 2, sizeof(int));
        p->freq[l] = (float*)calloc((size_t)nchan + 2, sizeof(float));
    }
    /* level 0: uniform channel edges in float, one delay span for all */
    float bw = fmax - fmin;
    float step = bw / (float)nchan;
    int d0 = delta_t(p, fmin, fmin + step);
    p->nsub[0] = nchan;
    for (int i = 0; i < nchan; ++i) {
        float v = (float)i * bw;
        p->freq[0][i] = fmin + v / (float)nchan;
        p->rows[0][i] = d0 + 1;
    }
    p->freq[0][nchan] = fmax;
    for (int l = 1; l <= p->niter; ++l) {
        int q = p->nsub[l - 1];
        const float* f = p->freq[l - 1];
        int half = q / 2, qn;
        for (int i = 0; i < half; ++i) {
            p->rows[l][i] = delta_t(p, f[2 * i], f[2 * i + 2]) + 1;
            p->freq[l][i] = f[2 * i];
        }
        if (q & 1) {
            qn = half + 1;
            p->freq[l][qn - 1] = f[q - 1];
            p->rows[l][qn - 1] = p->rows[l - 1][q - 1];
        } else {
            qn = half;
        }
        p->freq[l][qn] = fmax;
        p->nsub[l] = qn;
    }
    for (int l = 0; l <= p->niter; ++l) {
        p->cum[l][0] = 0;
        for (int i = 0; i < p->nsub[l]; ++i) p->cum[l][i + 1] = p->cum[l][i] + p->rows[l][i];
    }
    return 0;
}

int orc_fdmt_rows(float fmin, float fmax, int nchan, int max_dt, int* rows_per_level, int cap) {
    oplan p;
    if (plan_build(&p, fmin, fmax, nchan, max_dt)) { plan_free(&p); return -1; }
    for (int l = 0; l <= p.niter && l < cap; ++l) rows_per_level[l] = p.cum[l][p.nsub[l]];
    int n = p.niter;
    plan_free(&p);
    return n;
}

/* Row tables for level l >= 1 (global row indices in the previous plane). */
static int level_tables(const oplan* p, int l, int* a, int* b, int* s, int cap) {
    int qin = p->nsub[l - 1], qout = p->nsub[l];
    const int* cin = p->cum[l - 1];
    const int* cout = p->cum[l];
    const float* f = p->freq[l - 1];
    for (int i = 0; i < qout; ++i) {
        int r0 = cout[i], nr = cout[i + 1] - cout[i];
        if (2 * i + 1 >= qin) { /* odd count: the last sub-band is carried over */
            for (int j = 0; j < nr; ++j) {
                if (r0 + j < cap) { a[r0 + j] = cin[2 * i] + j; b[r0 + j] = -1; s[r0 + j] = 0; }
            }
            continue;
        }
        float dall = band_delay(f[2 * i], f[2 * i + 2]);
        float c0 = band_delay(f[2 * i], f[2 * i + 1]) / dall;
        float c1 = band_delay(f[2 * i + 1], f[2 * i + 2]) / dall;
        for (int j = 0; j < nr; ++j) {
            int j0 = (int)(c0 * (float)j);
            int j1 = (int)(c1 * (float)j);
            if (r0 + j < cap) { a[r0 + j] = cin[2 * i] + j0; b[r0 + j] = cin[2 * i + 1] + j1; s[r0 + j] = j0; }
        }
    }
    return cout[qout];
}

int orc_fdmt_tables(float fmin, float fmax, int nchan, int max_dt, int level,
                    int* a_row, int* b_row, int* shift, int cap) {
    oplan p;
    if (plan_build(&p, fmin, fmax, nchan, max_dt) || level < 0 || level > p.niter) { plan_free(&p); return -1; }
    int n;
    if (level == 0) {
        n = p.cum[0][p.nsub[0]];
    } else {
        n = level_tables(&p, level, a_row, b_row, shift, cap);
    }
    plan_free(&p);
    return n;
}

/* ---- reduced-precision planes -------------------------------------------
 * The value of the binary16 (IEEE 754 half: 11 significant bits, exponent
 * -14..15, subnormal quantum 2^-24) nearest to v, ties to even, as a float;
 * beyond the largest finite half (65504) rounding gives infinity.  Scaling a
 * float by a power of two is exact here, so the nearest multiple of the
 * quantum is taken with nearbyintf (round-to-nearest-even mode). */
static float round_f16(float v) {
    if (isnan(v)) return v;
    float a = fabsf(v);
    if (a >= 65520.0f) return copysignf(INFINITY, v);
    float q;
    if (a < 6.103515625e-05f) { /* 2^-14: subnormal halves */
        q = nearbyintf(a * 16777216.0f) / 16777216.0f;
    } else {
        int e;
        frexpf(a, &e); /* a = m 2^e, m in [0.5, 1): quantum 2^(e-11) */
        float sc = ldexpf(1.0f, 11 - e);
        q = nearbyintf(a * sc) / sc;
    }
    return copysignf(q, v);
}

/* bfloat16: the upper 16 bits of the float, rounded to nearest even. */
static float round_bf16(float v) {
    if (isnan(v)) return v;
    uint32_t u;
    memcpy(&u, &v, 4);
    u = (u + 0x7fffu + ((u >> 16) & 1u)) & 0xffff0000u;
    memcpy(&v, &u, 4);
    return v;
}

/* Plane of level l stored at 16 bits: row g keeps round(v * 2^-e_g) * 2^e_g,
 * e_g = ceil(log2(channels summed into row g)). */
static void round_plane(float* pl, int rows, int cols, const int* cnt, int prec) {
    for (int g = 0; g < rows; ++g) {
        int e = 0;
        while ((1 << e) < cnt[g]) ++e;
        float dn = ldexpf(1.0f, -e), up = ldexpf(1.0f, e);
        float* r = pl + (size_t)g * cols;
        for (int t = 0; t < cols; ++t) {
            float x = r[t] * dn;
            r[t] = (prec == ORC_PREC_BF16 ? round_bf16(x) : round_f16(x)) * up;
        }
    }
}

void orc_round16(const float* in, float* out, int64_t n, int prec) {
    for (int64_t i = 0; i < n; ++i) out[i] = prec == ORC_PREC_BF16 ? round_bf16(in[i]) : round_f16(in[i]);
}

#define NO_ROUND(pl, rows, cols, cnt, prec) ((void)0)
#define DO_ROUND(pl, rows, cols, cnt, prec) round_plane(pl, rows, cols, cnt, prec)

#define DEFINE_RUN(NAME, T, ROUND)                                                       \
static int NAME(float fmin, float fmax, int nchan, int cols, int max_dt,                 \
                const T* in, T* out, int b_ones, int prec, int kstore) {                 \
    oplan p;                                                                             \
    if (plan_build(&p, fmin, fmax, nchan, max_dt) || cols < 1) { plan_free(&p); return -1; } \
    int maxr[2] = {0, 0};                                                                \
    for (int l = 0; l <= p.niter; ++l) {                                                 \
        int r = p.cum[l][p.nsub[l]];                                                     \
        if (r > maxr[l & 1]) maxr[l & 1] = r;                                            \
    }                                                                                    \
    if (p.cum[p.niter][p.nsub[p.niter]] != max_dt) { plan_free(&p); return -2; }         \
    T* pl[2];                                                                            \
    pl[0] = (T*)calloc((size_t)maxr[0] * cols, sizeof(T));                               \
    pl[1] = (T*)calloc((size_t)(maxr[1] > 0 ? maxr[1] : 1) * cols, sizeof(T));          \
    int nr0 = p.rows[0][0];                                                              \
    int* cnt[2];                                 /* channels summed per row */           \
    cnt[0] = (int*)malloc(sizeof(int) * (size_t)(maxr[0] > maxr[1] ? maxr[0] : maxr[1]) + 4); \
    cnt[1] = (int*)malloc(sizeof(int) * (size_t)(maxr[0] > maxr[1] ? maxr[0] : maxr[1]) + 4); \
    for (int g = 0; g < nchan * nr0; ++g) cnt[0][g] = 1;                                 \
    /* level 0: row r of channel c is the running mean of x[t-r..t]; 0 for t < r */      \
    for (int c = 0; c < nchan; ++c) {                                                    \
        T* base = pl[0] + (size_t)c * nr0 * cols;                                        \
        for (int t = 0; t < cols; ++t) base[t] = b_ones ? (T)1 : in[(size_t)c * cols + t]; \
        for (int r = 1; r < nr0; ++r) {                                                  \
            T* cur = base + (size_t)r * cols;                                            \
            const T* prev = cur - cols;                                                  \
            for (int t = 0; t < cols; ++t) {                                             \
                if (t < r) { cur[t] = 0; continue; }                                     \
                T x = b_ones ? (T)1 : in[(size_t)c * cols + t - r];                      \
                T m = prev[t] * (T)r;                                                    \
                T sum = m + x;                                                           \
                cur[t] = sum / (T)(r + 1);                                               \
            }                                                                            \
        }                                                                                \
    }                                                                                    \
    if (prec && kstore == 0 && p.niter > 0) ROUND(pl[0], nchan * nr0, cols, cnt[0], prec); \
    int rmax = 0;                                                                        \
    for (int l = 1; l <= p.niter; ++l) { int r = p.cum[l][p.nsub[l]]; if (r > rmax) rmax = r; } \
    int* a = (int*)malloc(sizeof(int) * (rmax + 1));                                     \
    int* b = (int*)malloc(sizeof(int) * (rmax + 1));                                     \
    int* s = (int*)malloc(sizeof(int) * (rmax + 1));                                     \
    for (int l = 1; l <= p.niter; ++l) {                                                 \
        const T* src = pl[(l - 1) & 1];                                                  \
        T* dst = pl[l & 1];                                                              \
        int nr = level_tables(&p, l, a, b, s, rmax + 1);                                 \
        for (int g = 0; g < nr; ++g) {                                                   \
            const T* ra = src + (size_t)a[g] * cols;                                     \
            T* ro = dst + (size_t)g * cols;                                              \
            cnt[l & 1][g] = cnt[(l - 1) & 1][a[g]] + (b[g] >= 0 ? cnt[(l - 1) & 1][b[g]] : 0); \
            if (b[g] < 0) { memcpy(ro, ra, sizeof(T) * cols); continue; }                \
            const T* rb = src + (size_t)b[g] * cols;                                     \
            int sh = s[g];                                                               \
            for (int t = 0; t < cols; ++t) ro[t] = (t >= sh) ? ra[t] + rb[t - sh] : ra[t]; \
        }                                                                                \
        if (prec && l >= kstore && l < p.niter) ROUND(dst, nr, cols, cnt[l & 1], prec);  \
    }                                                                                    \
    memcpy(out, pl[p.niter & 1], sizeof(T) * (size_t)max_dt * cols);                    \
    free(a); free(b); free(s); free(pl[0]); free(pl[1]); free(cnt[0]); free(cnt[1]);     \
    plan_free(&p);                                                                       \
    return 0;                                                                            \
}

DEFINE_RUN(run_f32, float, DO_ROUND)
DEFINE_RUN(run_f64, double, NO_ROUND)

int orc_fdmt_run_f32(float fmin, float fmax, int nchan, int cols, int max_dt,
                     const float* in, float* out, int b_ones) {
    return run_f32(fmin, fmax, nchan, cols, max_dt, in, out, b_ones, 0, 0);
}

int orc_fdmt_run_f64(float fmin, float fmax, int nchan, int cols, int max_dt,
                     const double* in, double* out, int b_ones) {
    return run_f64(fmin, fmax, nchan, cols, max_dt, in, out, b_ones, 0, 0);
}

int orc_fdmt_run_lowp(float fmin, float fmax, int nchan, int cols, int max_dt,
                      const float* in, float* out, int b_ones, int prec, int kstore) {
    if (prec != ORC_PREC_F16 && prec != ORC_PREC_BF16) return -3;
    return run_f32(fmin, fmax, nchan, cols, max_dt, in, out, b_ones, prec, kstore);
}

/* ---- adjoint --------------------------------------------------------------
 * Transpose of the FDMT (the product's adjoint, no reference counterpart):
 *   merge level l: gin[i][u] = sum, over the level-l rows g that read row i
 *     (as tail a_g, shift 0, or head b_g, shift s_g) in ascending g, of
 *     gout[g][u + shift] where u + shift < cols;
 *   level 0: gx[c][u] = sum_{r'} RN(1/(r'+1)) * sum_{r=0..r'} [u+r >= r'][u+r < cols]
 *     g0[c,r'][u+r] (inner sums r ascending, outer r' ascending).
 * With T = float the sums run in exactly that order. */
#define DEFINE_ADJ(NAME, T)                                                              \
int NAME(float fmin, float fmax, int nchan, int cols, int max_dt, const T* gy, T* gx) {  \
    oplan p;                                                                             \
    if (plan_build(&p, fmin, fmax, nchan, max_dt) || cols < 1) { plan_free(&p); return -1; } \
    if (p.cum[p.niter][p.nsub[p.niter]] != max_dt) { plan_free(&p); return -2; }         \
    int rmax = 0;                                                                        \
    for (int l = 0; l <= p.niter; ++l) { int r = p.cum[l][p.nsub[l]]; if (r > rmax) rmax = r; } \
    T* cur = (T*)malloc(sizeof(T) * (size_t)max_dt * cols);                              \
    memcpy(cur, gy, sizeof(T) * (size_t)max_dt * cols);                                  \
    int* a = (int*)malloc(sizeof(int) * (rmax + 1));                                     \
    int* b = (int*)malloc(sizeof(int) * (rmax + 1));                                     \
    int* s = (int*)malloc(sizeof(int) * (rmax + 1));                                     \
    int* cnt = (int*)malloc(sizeof(int) * (rmax + 2));                                   \
    int* eg = (int*)malloc(sizeof(int) * 2 * (rmax + 1));                                \
    int* es = (int*)malloc(sizeof(int) * 2 * (rmax + 1));                                \
    for (int l = p.niter; l >= 1; --l) {                                                 \
        int nout = level_tables(&p, l, a, b, s, rmax + 1);                               \
        int nin = p.cum[l - 1][p.nsub[l - 1]];                                           \
        for (int i = 0; i <= nin; ++i) cnt[i] = 0;                                       \
        for (int g = 0; g < nout; ++g) { ++cnt[a[g] + 1]; if (b[g] >= 0) ++cnt[b[g] + 1]; } \
        for (int i = 0; i < nin; ++i) cnt[i + 1] += cnt[i];                              \
        int* fill = (int*)malloc(sizeof(int) * ((size_t)nin + 1));                       \
        memcpy(fill, cnt, sizeof(int) * (nin + 1));                                      \
        for (int g = 0; g < nout; ++g) {                                                 \
            int k = fill[a[g]]++; eg[k] = g; es[k] = 0;                                  \
            if (b[g] >= 0) { k = fill[b[g]]++; eg[k] = g; es[k] = s[g]; }                \
        }                                                                                \
        T* nxt = (T*)calloc((size_t)(unsigned)nin * (size_t)(unsigned)cols, sizeof(T));  \
        for (int i = 0; i < nin; ++i) {                                                  \
            T* o = nxt + (size_t)i * cols;                                               \
            for (int k = cnt[i]; k < cnt[i + 1]; ++k) {                                  \
                const T* src = cur + (size_t)eg[k] * cols;                               \
                int sh = es[k];                                                          \
                for (int u = 0; u + sh < cols; ++u) o[u] = o[u] + src[u + sh];          \
            }                                                                            \
        }                                                                                \
        free(fill); free(cur); cur = nxt;                                                \
    }                                                                                    \
    int R = p.rows[0][0];                                                                \
    for (int c = 0; c < nchan; ++c) {                                                    \
        const T* g0 = cur + (size_t)c * R * cols;                                        \
        for (int u = 0; u < cols; ++u) {                                                 \
            T acc = 0;                                                                   \
            for (int rr = 0; rr < R; ++rr) {                                             \
                T w = 0;                                                                 \
                for (int r = 0; r <= rr; ++r) {                                          \
                    int t = u + r;                                                       \
                    if (t >= rr && t < cols) w = w + g0[(size_t)rr * cols + t];          \
                }                                                                        \
                acc = acc + w * ((T)1 / (T)(rr + 1));                                    \
            }                                                                            \
            gx[(size_t)c * cols + u] = acc;                                              \
        }                                                                                \
    }                                                                                    \
    free(cur); free(a); free(b); free(s); free(cnt); free(eg); free(es);                 \
    plan_free(&p);                                                                       \
    return 0;                                                                            \
}

DEFINE_ADJ(orc_fdmt_adjoint_f32, float)
DEFINE_ADJ(orc_fdmt_adjoint_f64, double)
