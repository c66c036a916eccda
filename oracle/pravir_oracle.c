/* ORACLE — test infrastructure only (see oracle.h).
 *
 * Restatement of the reference's second FDMT variant (the "Pravir" plan),
 * single threaded:
 *   plan      MyVSLib_C++/FDMT_PRAVIR/fdmt_base.cpp:86-104 (niters, df, dt
 *             grid of a sub-band), :139-172 (level 0), :174-278 (levels >= 1:
 *             sub-band edges, mid-band dt mappings, head/tail/offset, copies)
 *   helpers   MyVSLib_C++/FDMT_PRAVIR/fdmtUtils.cpp:36-45 (cff, dt of a
 *             sub-band), :92-108 (closest index in a dt grid)
 *   level 0   MyVSLib_C++/FDMT_PRAVIR/fdmt_cpu.cpp:103-179 (window means)
 *   level i   MyVSLib_C++/FDMT_PRAVIR/fdmt_cpu.cpp:243-301 with
 *             fdmtUtils.cpp:47-90 (tail + offset head, copies)
 * Float expressions keep the reference's types (float band edges and
 * coefficients from powf, roundf to the dt grid), so with -ffp-contract=off
 * the FP32 result is bit-identical to a fresh FDMTCPU object's execute().
 * Samples a level-0 row does not define (t < dt) are 0, as in that object.
 */
#include "oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define PMAXL 40

typedef struct {
    int niter;
    int nsub[PMAXL];
    int* cum[PMAXL];   /* nsub+1 cumulative rows                    */
    int* dt[PMAXL];    /* dt value of every row (level 0 and all)   */
    int* a[PMAXL];     /* level >= 1: tail row (global), per row     */
    int* b[PMAXL];     /* head row (global) or -1 for a copied row  */
    int* s[PMAXL];     /* offset                                    */
} pplan;

static float cff(float f1s, float f1e, float f2s, float f2e) {
    return (powf(f1s, -2.0f) - powf(f1e, -2.0f)) / (powf(f2s, -2.0f) - powf(f2e, -2.0f));
}

static long dt_sub(float fs, float fe, float fmin, float fmax, long dt) {
    float ratio = cff(fs, fe, fmin, fmax);
    return (long)roundf((float)dt * ratio);
}

/* dt grid of a sub-band into g (cap entries); returns its length */
static int grid_sub(float fs, float fe, float fmin, float fmax, long dt_max, long dt_min, long step,
                    int* g, int cap) {
    long hi = dt_sub(fs, fe, fmin, fmax, dt_max), lo = dt_sub(fs, fe, fmin, fmax, dt_min);
    int n = 0;
    for (long d = lo; d <= hi; d += step) {
        if (n < cap) g[n] = (int)d;
        ++n;
    }
    return n;
}

static int closest(const int* g, int n, long val) {
    int lo = 0, hi = n; /* lower bound */
    while (lo < hi) { int m = (lo + hi) / 2; if (g[m] < val) lo = m + 1; else hi = m; }
    int idx = lo;
    if (lo < n) {
        if (lo > 0 && val - g[lo - 1] < g[lo] - val) idx = lo - 1;
    } else {
        idx = n - 1;
    }
    return idx;
}

static void pplan_free(pplan* p) {
    for (int l = 0; l < PMAXL; ++l) { free(p->cum[l]); free(p->dt[l]); free(p->a[l]); free(p->b[l]); free(p->s[l]); }
    memset(p, 0, sizeof(*p));
}

/* Returns 0, or < 0 where the reference throws (a mid-band dt above dt, an
 * offset >= nsamps, an empty grid). */
static int pplan_build(pplan* p, float fmin, float fmax, int nchans, int nsamps, long dt_max,
                       long dt_step, long dt_min) {
    memset(p, 0, sizeof(*p));
    if (nchans < 1 || nsamps < 1 || dt_step < 1 || !(fmax > fmin)) return -1;
    int niter = 0;
    while ((1L << niter) < nchans) ++niter;
    if (niter + 1 > PMAXL) return -1;
    p->niter = niter;
    const float df = (fmax - fmin) / (float)nchans;
    const float corr = df / 2;
    const int cap = (int)((dt_max - dt_min) / dt_step + 2);
    /* level 0 */
    p->nsub[0] = nchans;
    p->cum[0] = (int*)calloc((size_t)nchans + 1, sizeof(int));
    int* tmp = (int*)malloc(sizeof(int) * (size_t)cap);
    int** g0 = (int**)calloc((size_t)nchans, sizeof(int*));
    int* n0 = (int*)calloc((size_t)nchans, sizeof(int));
    for (int i = 0; i < nchans; ++i) {
        float fs = df * (float)i + fmin;
        float fe = fs + df;
        n0[i] = grid_sub(fs, fe, fmin, fmax, dt_max, dt_min, dt_step, tmp, cap);
        if (n0[i] <= 0) { free(tmp); for (int k = 0; k < nchans; ++k) free(g0[k]); free(g0); free(n0); pplan_free(p); return -3; }
        g0[i] = (int*)malloc(sizeof(int) * (size_t)n0[i]);
        memcpy(g0[i], tmp, sizeof(int) * (size_t)n0[i]);
        p->cum[0][i + 1] = p->cum[0][i] + n0[i];
    }
    p->dt[0] = (int*)malloc(sizeof(int) * (size_t)p->cum[0][nchans]);
    for (int i = 0; i < nchans; ++i) memcpy(p->dt[0] + p->cum[0][i], g0[i], sizeof(int) * (size_t)n0[i]);
    /* grids of the previous level's sub-bands, and the top sub-band grid */
    int** gp = g0; int* np = n0;
    int* gtop = (int*)malloc(sizeof(int) * (size_t)n0[nchans - 1]);
    int ntop = n0[nchans - 1];
    memcpy(gtop, g0[nchans - 1], sizeof(int) * (size_t)ntop);
    float df_top = df, df_bot = df;
    int rc = 0;
    for (int l = 1; l <= niter && rc == 0; ++l) {
        const int nprev = p->nsub[l - 1];
        const int ncur = nprev / 2 + nprev % 2;
        const int do_copy = nprev % 2 == 1;
        const float dtop = do_copy ? df_top : df_top + df_bot;
        const float dbot = df_bot * 2;
        p->nsub[l] = ncur;
        p->cum[l] = (int*)calloc((size_t)ncur + 1, sizeof(int));
        int** gc = (int**)calloc((size_t)ncur, sizeof(int*));
        int* nc = (int*)calloc((size_t)ncur, sizeof(int));
        /* rows of every sub-band first (grids), then the tables */
        float* fst = (float*)malloc(sizeof(float) * (size_t)ncur);
        float* fen = (float*)malloc(sizeof(float) * (size_t)ncur);
        float* fmd = (float*)malloc(sizeof(float) * (size_t)ncur);
        for (int i = 0; i < ncur; ++i) {
            float fs = dbot * (float)i + fmin, fe, fm;
            if (i == ncur - 1) {
                if (do_copy) {
                    fe = fs + dtop * 2;
                    fm = fs + dtop;
                    nc[i] = ntop;
                    gc[i] = (int*)malloc(sizeof(int) * (size_t)ntop);
                    memcpy(gc[i], gtop, sizeof(int) * (size_t)ntop);
                } else {
                    fe = fs + dtop;
                    fm = fs + dbot / 2;
                    nc[i] = grid_sub(fs, fe, fmin, fmax, dt_max, dt_min, dt_step, tmp, cap);
                    gc[i] = (int*)malloc(sizeof(int) * (size_t)(nc[i] > 0 ? nc[i] : 1));
                    memcpy(gc[i], tmp, sizeof(int) * (size_t)nc[i]);
                    free(gtop);
                    ntop = nc[i];
                    gtop = (int*)malloc(sizeof(int) * (size_t)(ntop > 0 ? ntop : 1));
                    memcpy(gtop, tmp, sizeof(int) * (size_t)ntop);
                }
            } else {
                fe = fs + dbot;
                fm = fs + dbot / 2;
                nc[i] = grid_sub(fs, fe, fmin, fmax, dt_max, dt_min, dt_step, tmp, cap);
                gc[i] = (int*)malloc(sizeof(int) * (size_t)(nc[i] > 0 ? nc[i] : 1));
                memcpy(gc[i], tmp, sizeof(int) * (size_t)nc[i]);
            }
            if (nc[i] <= 0) rc = -3;
            fst[i] = fs; fen[i] = fe; fmd[i] = fm;
            p->cum[l][i + 1] = p->cum[l][i] + nc[i];
        }
        const int rows = p->cum[l][ncur];
        p->dt[l] = (int*)malloc(sizeof(int) * (size_t)(rows > 0 ? rows : 1));
        p->a[l] = (int*)malloc(sizeof(int) * (size_t)(rows > 0 ? rows : 1));
        p->b[l] = (int*)malloc(sizeof(int) * (size_t)(rows > 0 ? rows : 1));
        p->s[l] = (int*)malloc(sizeof(int) * (size_t)(rows > 0 ? rows : 1));
        for (int i = 0; i < ncur && rc == 0; ++i) {
            const int tail = 2 * i, head = 2 * i + 1;
            const float fs = fst[i], fe = fen[i];
            const float fm1 = fmd[i] - corr, fm2 = fmd[i] + corr;
            for (int j = 0; j < nc[i]; ++j) {
                const long dt = gc[i][j];
                const long m1 = (long)roundf((float)dt * cff(fs, fm1, fs, fe));
                const long m2 = (long)roundf((float)dt * cff(fs, fm2, fs, fe));
                if (m1 > dt || m2 > dt) { rc = -4; break; }
                const int row = p->cum[l][i] + j;
                p->dt[l][row] = (int)dt;
                if (i == ncur - 1 && do_copy) {
                    p->a[l][row] = p->cum[l - 1][tail] + closest(gp[tail], np[tail], dt);
                    p->b[l][row] = -1;
                    p->s[l][row] = 0;
                } else {
                    if (m2 >= nsamps) { rc = -5; break; }
                    p->a[l][row] = p->cum[l - 1][tail] + closest(gp[tail], np[tail], m1);
                    p->b[l][row] = p->cum[l - 1][head] + closest(gp[head], np[head], dt - m2);
                    p->s[l][row] = (int)m2;
                }
            }
        }
        free(fst); free(fen); free(fmd);
        for (int k = 0; k < nprev; ++k) free(gp[k]);
        free(gp); free(np);
        gp = gc; np = nc;
        df_top = dtop; df_bot = dbot;
    }
    for (int k = 0; k < p->nsub[niter]; ++k) free(gp[k]);
    free(gp); free(np); free(gtop); free(tmp);
    if (rc != 0) pplan_free(p);
    return rc;
}

static int level_rows(const pplan* p, int l) { return p->cum[l][p->nsub[l]]; }

int orc_pravir_rows(float fmin, float fmax, int nchans, int nsamps, long dt_max, long dt_step,
                    long dt_min, int* rows_per_level, int cap) {
    pplan p;
    int rc = pplan_build(&p, fmin, fmax, nchans, nsamps, dt_max, dt_step, dt_min);
    if (rc) return rc;
    for (int l = 0; l <= p.niter && l < cap; ++l) rows_per_level[l] = level_rows(&p, l);
    int n = p.niter;
    pplan_free(&p);
    return n;
}

int orc_pravir_level(float fmin, float fmax, int nchans, int nsamps, long dt_max, long dt_step,
                     long dt_min, int level, int* cum, int* dt, int* a_row, int* b_row, int* shift,
                     int cap) {
    pplan p;
    int rc = pplan_build(&p, fmin, fmax, nchans, nsamps, dt_max, dt_step, dt_min);
    if (rc) return rc;
    if (level < 0 || level > p.niter) { pplan_free(&p); return -1; }
    const int rows = level_rows(&p, level);
    if (cum) for (int i = 0; i <= p.nsub[level] && i < cap; ++i) cum[i] = p.cum[level][i];
    for (int r = 0; r < rows && r < cap; ++r) {
        if (dt) dt[r] = p.dt[level][r];
        if (level > 0) {
            if (a_row) a_row[r] = p.a[level][r];
            if (b_row) b_row[r] = p.b[level][r];
            if (shift) shift[r] = p.s[level][r];
        }
    }
    pplan_free(&p);
    return rows;
}

#define DEFINE_PRUN(NAME, T)                                                              \
int NAME(float fmin, float fmax, int nchans, int nsamps, long dt_max, long dt_step,      \
         long dt_min, const T* in, T* out) {                                              \
    pplan p;                                                                              \
    int rc = pplan_build(&p, fmin, fmax, nchans, nsamps, dt_max, dt_step, dt_min);        \
    if (rc) return rc;                                                                    \
    int rmax = 0;                                                                         \
    for (int l = 0; l <= p.niter; ++l) if (level_rows(&p, l) > rmax) rmax = level_rows(&p, l); \
    T* cur = (T*)calloc((size_t)rmax * (size_t)nsamps, sizeof(T));                        \
    T* nxt = (T*)calloc((size_t)rmax * (size_t)nsamps, sizeof(T));                        \
    for (int c = 0; c < nchans; ++c) {                                                    \
        const T* x = in + (size_t)c * nsamps;                                             \
        const int r0 = p.cum[0][c], nr = p.cum[0][c + 1] - r0;                            \
        const int* dts = p.dt[0] + r0;                                                    \
        T* row = cur + (size_t)r0 * nsamps;                                               \
        for (int t = dts[0]; t < nsamps; ++t) {                                           \
            T sum = 0;                                                                    \
            for (int i = t - dts[0]; i <= t; ++i) sum += x[i];                            \
            row[t] = sum / (T)(dts[0] + 1);                                               \
        }                                                                                 \
        for (int k = 1; k < nr; ++k) {                                                    \
            T* rk = cur + (size_t)(r0 + k) * nsamps;                                      \
            const T* rp = rk - nsamps;                                                    \
            for (int t = dts[k]; t < nsamps; ++t) {                                       \
                T sum = 0;                                                                \
                for (int i = t - dts[k]; i < t - dts[k - 1]; ++i) sum += x[i];            \
                rk[t] = (rp[t] * ((T)dts[k - 1] + (T)1) + sum) / ((T)dts[k] + (T)1);      \
            }                                                                             \
        }                                                                                 \
    }                                                                                     \
    for (int l = 1; l <= p.niter; ++l) {                                                  \
        const int rows = level_rows(&p, l);                                               \
        for (int g = 0; g < rows; ++g) {                                                  \
            const T* ta = cur + (size_t)p.a[l][g] * nsamps;                               \
            T* o = nxt + (size_t)g * nsamps;                                              \
            if (p.b[l][g] < 0) { memcpy(o, ta, sizeof(T) * (size_t)nsamps); continue; }   \
            const T* hb = cur + (size_t)p.b[l][g] * nsamps;                               \
            const int off = p.s[l][g];                                                    \
            for (int t = 0; t < nsamps; ++t) o[t] = t >= off ? ta[t] + hb[t - off] : ta[t]; \
        }                                                                                 \
        T* sw = cur; cur = nxt; nxt = sw;                                                 \
    }                                                                                     \
    memcpy(out, cur, sizeof(T) * (size_t)level_rows(&p, p.niter) * (size_t)nsamps);       \
    free(cur); free(nxt);                                                                 \
    pplan_free(&p);                                                                       \
    return 0;                                                                             \
}

DEFINE_PRUN(orc_pravir_run_f32, float)
DEFINE_PRUN(orc_pravir_run_f64, double)

/* Adjoint: merge levels as gathers over the readers of each row in
 * ascending output row, then level 0 as
 *   gx[c][u] = sum_k RN(1/(dt_k+1)) * sum_{j=0..dt_k} [u+j >= dt_k][u+j < nsamps] g0[k][u+j]
 * (the window mean's transpose; inner sums j ascending, outer k ascending). */
#define DEFINE_PADJ(NAME, T)                                                              \
int NAME(float fmin, float fmax, int nchans, int nsamps, long dt_max, long dt_step,      \
         long dt_min, const T* gy, T* gx) {                                               \
    pplan p;                                                                              \
    int rc = pplan_build(&p, fmin, fmax, nchans, nsamps, dt_max, dt_step, dt_min);        \
    if (rc) return rc;                                                                    \
    int rmax = 0;                                                                         \
    for (int l = 0; l <= p.niter; ++l) if (level_rows(&p, l) > rmax) rmax = level_rows(&p, l); \
    T* cur = (T*)calloc((size_t)rmax * (size_t)nsamps, sizeof(T));                        \
    T* nxt = (T*)calloc((size_t)rmax * (size_t)nsamps, sizeof(T));                        \
    memcpy(cur, gy, sizeof(T) * (size_t)level_rows(&p, p.niter) * (size_t)nsamps);        \
    for (int l = p.niter; l >= 1; --l) {                                                  \
        const int nin = level_rows(&p, l - 1), nout = level_rows(&p, l);                  \
        memset(nxt, 0, sizeof(T) * (size_t)nin * (size_t)nsamps);                         \
        /* ascending g: every input row receives its terms in ascending g */              \
        for (int g = 0; g < nout; ++g) {                                                  \
            const T* src = cur + (size_t)g * nsamps;                                      \
            T* oa = nxt + (size_t)p.a[l][g] * nsamps;                                     \
            for (int u = 0; u < nsamps; ++u) oa[u] = oa[u] + src[u];                      \
            if (p.b[l][g] >= 0) {                                                         \
                T* ob = nxt + (size_t)p.b[l][g] * nsamps;                                 \
                const int sh = p.s[l][g];                                                 \
                for (int u = 0; u + sh < nsamps; ++u) ob[u] = ob[u] + src[u + sh];        \
            }                                                                             \
        }                                                                                 \
        T* sw = cur; cur = nxt; nxt = sw;                                                 \
    }                                                                                     \
    for (int c = 0; c < nchans; ++c) {                                                    \
        const int r0 = p.cum[0][c], nr = p.cum[0][c + 1] - r0;                            \
        for (int u = 0; u < nsamps; ++u) {                                                \
            T acc = 0;                                                                    \
            for (int k = 0; k < nr; ++k) {                                                \
                const int d = p.dt[0][r0 + k];                                            \
                const T* g0 = cur + (size_t)(r0 + k) * nsamps;                            \
                T w = 0;                                                                  \
                for (int j = 0; j <= d; ++j) {                                            \
                    const int t = u + j;                                                  \
                    if (t >= d && t < nsamps) w = w + g0[t];                              \
                }                                                                         \
                acc = acc + w * ((T)1 / (T)(d + 1));                                      \
            }                                                                             \
            gx[(size_t)c * nsamps + u] = acc;                                             \
        }                                                                                 \
    }                                                                                     \
    free(cur); free(nxt);                                                                 \
    pplan_free(&p);                                                                       \
    return 0;                                                                             \
}

DEFINE_PADJ(orc_pravir_adjoint_f32, float)
DEFINE_PADJ(orc_pravir_adjoint_f64, double)
