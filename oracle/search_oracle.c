/* ORACLE — test infrastructure only (see oracle.h).
 *
 * Restatement of the reference's detection / clustering / normalisation:
 *   orc_boxcar            MyVSLib_C++/Clusterization/Clusterization.cu:420-455
 *                         (mode 0, widths 1,2,4..2^Q, mwidth = log2 w) and
 *                         :592-671 (mode 1, widths 1..W, mwidth = w); the
 *                         window sum is sequential from the start sample and
 *                         only complete windows are tested.  The S/N is the
 *                         IEEE quotient sum / sqrtf(w).
 *   orc_cluster           MyVSLib_C++/Clusterization/Clusterization.cu:92-166
 *                         (three passes mt, mdt, mwidth; sort inside each
 *                         group, split where consecutive keys differ by more
 *                         than the metric, :855-893 / :931-998), then
 *   orc_select_delegates  MyVSLib_C++/Clusterization/select_delegates.cu:63-125
 *                         (per-group argmax of msnr with a strided scan of
 *                         `block` lanes and a lowest-lane-wins reduction), and
 *                         the delegate sort by mt (Clusterization.cu:147-149).
 *   orc_calc_fdmt_inputs  MyVSLib_C++/CDMT/Statistical_preprocessing.cu:15-88
 *                         (row mean/variance, global mean/std, 4-sigma zap of
 *                         rows by variance, (x-mean)/std, ones mask).
 *   orc_norm_rows         per-delay-row (x - mean_r) / std_r of a DM-time
 *                         plane; the reference has no such routine, this is
 *                         the definition the product implements.
 * Ordering: the reference's sorts are unstable (cub segmented sort, thrust
 * sort); the restatement breaks every tie by candidate index, the canonical
 * order the product also uses.
 */
#include "oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

int64_t orc_boxcar(const float* plane, int rows, int cols, float thr, int mode,
                   int param, orc_cand* out, int64_t cap) {
    int64_t n = 0;
    int wmax = (mode == 0) ? (1 << param) : param;
    for (int r = 0; r < rows; ++r) {
        const float* row = plane + (size_t)r * cols;
        for (int t = 0; t < cols; ++t) {
            float sum = 0.0f;
            int next_pow = 1, pw = 0;
            for (int w = 1; w <= wmax; ++w) {
                if (t + w - 1 >= cols) break;
                sum = sum + row[t + w - 1];
                int emit = 0, width_code = w;
                if (mode == 0) {
                    if (w == next_pow) { emit = 1; width_code = pw; ++pw; next_pow *= 2; }
                } else {
                    emit = 1;
                }
                if (!emit) continue;
                float s = sum / sqrtf((float)w);
                if (s > thr) {
                    if (n < cap) { out[n].mt = t; out[n].mdt = r; out[n].mwidth = width_code; out[n].msnr = s; }
                    ++n;
                }
            }
        }
    }
    return n;
}

/* Same result as orc_boxcar (row-major order), rows split across OpenMP
 * threads; used to time the CPU baseline on many cores. */
int64_t orc_boxcar_mt(const float* plane, int rows, int cols, float thr, int mode,
                      int param, orc_cand* out, int64_t cap) {
    int64_t* cnt = (int64_t*)calloc((size_t)rows + 1, sizeof(int64_t));
    #pragma omp parallel for schedule(dynamic, 4)
    for (int r = 0; r < rows; ++r)
        cnt[r + 1] = orc_boxcar(plane + (size_t)r * cols, 1, cols, thr, mode, param, NULL, 0);
    for (int r = 0; r < rows; ++r) cnt[r + 1] += cnt[r];
    int64_t total = cnt[rows];
    if (total <= cap) {
        #pragma omp parallel for schedule(dynamic, 4)
        for (int r = 0; r < rows; ++r) {
            orc_cand* o = out + cnt[r];
            int64_t n = orc_boxcar(plane + (size_t)r * cols, 1, cols, thr, mode, param, o, cnt[r + 1] - cnt[r]);
            for (int64_t i = 0; i < n; ++i) o[i].mdt = r;
        }
    }
    free(cnt);
    return total;
}

void orc_norm_rows(const float* in, float* out, int rows, int cols, float* mean_out, float* std_out) {
    for (int r = 0; r < rows; ++r) {
        const float* x = in + (size_t)r * cols;
        double s = 0.0, ss = 0.0;
        for (int t = 0; t < cols; ++t) { double v = x[t]; s += v; ss += v * v; }
        double mean = s / cols;
        double var = ss / cols - mean * mean;
        if (var < 0) var = 0;
        float mf = (float)mean, sf = (float)sqrt(var);
        if (mean_out) mean_out[r] = mf;
        if (std_out) std_out[r] = sf;
        float* y = out + (size_t)r * cols;
        for (int t = 0; t < cols; ++t) {
            float d = x[t] - mf;
            y[t] = (sf > 0.0f) ? d / sf : 0.0f;
        }
    }
}

/* ---- clustering ---------------------------------------------------------- */
static const orc_cand* g_c;
static const int* g_gid;
static int g_field;

static int key_of(const orc_cand* c, int field) {
    return field == 0 ? c->mt : (field == 1 ? c->mdt : c->mwidth);
}

static int cmp_pass(const void* pa, const void* pb) {
    int a = *(const int*)pa, b = *(const int*)pb;
    if (g_gid[a] != g_gid[b]) return g_gid[a] < g_gid[b] ? -1 : 1;
    int ka = key_of(&g_c[a], g_field), kb = key_of(&g_c[b], g_field);
    if (ka != kb) return ka < kb ? -1 : 1;
    return a < b ? -1 : (a > b);
}

int orc_select_delegates(const orc_cand* c, const int* perm, const int* offsets,
                         int ngroups, int block, int* delegates) {
    float* v = (float*)malloc(sizeof(float) * (size_t)block);
    int* id = (int*)malloc(sizeof(int) * (size_t)block);
    for (int g = 0; g < ngroups; ++g) {
        int beg = offsets[g], len = offsets[g + 1] - offsets[g];
        for (int lane = 0; lane < block; ++lane) {
            v[lane] = -FLT_MAX;
            id[lane] = lane;  /* the reference stores the lane id for idle lanes */
            if (lane < len) {
                id[lane] = -1;
                for (int i = lane; i < len; i += block) {
                    int k = perm[beg + i];
                    if (c[k].msnr > v[lane]) { v[lane] = c[k].msnr; id[lane] = k; }
                }
            }
        }
        /* the reference's tree reduction: lane l takes lane l+s only if strictly
         * greater; on ties the winner follows the tree, not the lowest lane */
        for (int s = block / 2; s > 0; s >>= 1)
            for (int lane = 0; lane < s; ++lane)
                if (v[lane + s] > v[lane]) { v[lane] = v[lane + s]; id[lane] = id[lane + s]; }
        delegates[g] = id[0];
    }
    free(v);
    free(id);
    return ngroups;
}

static const orc_cand* g_dc;
static const int* g_dgroup;
static int cmp_deleg(const void* pa, const void* pb) {
    int a = *(const int*)pa, b = *(const int*)pb;  /* positions in group order */
    int ma = g_dc[g_dgroup[a]].mt, mb = g_dc[g_dgroup[b]].mt;
    if (ma != mb) return ma < mb ? -1 : 1;
    return a < b ? -1 : (a > b);
}

int orc_cluster(const orc_cand* c, int n, const int* metrics, int* perm_out,
                int* offsets_out, int* delegates_out) {
    if (n <= 0) { offsets_out[0] = 0; return 0; }
    int* gid = (int*)calloc((size_t)n, sizeof(int));
    int* perm = (int*)malloc(sizeof(int) * (size_t)n);
    int ngroups = 1;
    for (int field = 0; field < 3; ++field) {
        for (int i = 0; i < n; ++i) perm[i] = i;
        g_c = c; g_gid = gid; g_field = field;
        qsort(perm, (size_t)n, sizeof(int), cmp_pass);
        int cur = -1;
        for (int i = 0; i < n; ++i) {
            int k = perm[i];
            int split = (i == 0);
            if (!split) {
                int p = perm[i - 1];
                if (gid[p] != gid[k]) split = 1;
                else if ((long)key_of(&c[k], field) - (long)key_of(&c[p], field) > (long)metrics[field]) split = 1;
            }
            if (split) ++cur;
            perm_out[i] = cur;  /* temporary: new group id by position */
        }
        for (int i = 0; i < n; ++i) gid[perm[i]] = perm_out[i];
        ngroups = cur + 1;
    }
    /* final order and offsets */
    for (int i = 0; i < n; ++i) perm_out[i] = perm[i];
    int g = 0;
    offsets_out[0] = 0;
    for (int i = 1; i < n; ++i) if (gid[perm[i]] != gid[perm[i - 1]]) offsets_out[++g] = i;
    offsets_out[ngroups] = n;
    int* dl = (int*)malloc(sizeof(int) * (size_t)ngroups);
    orc_select_delegates(c, perm, offsets_out, ngroups, 64, dl);
    int* pos = (int*)malloc(sizeof(int) * (size_t)ngroups);
    for (int i = 0; i < ngroups; ++i) pos[i] = i;
    g_dc = c; g_dgroup = dl;
    qsort(pos, (size_t)ngroups, sizeof(int), cmp_deleg);
    for (int i = 0; i < ngroups; ++i) delegates_out[i] = dl[pos[i]];
    free(pos); free(dl); free(gid); free(perm);
    return ngroups;
}

/* ---- statistical preprocessing ------------------------------------------ */
void orc_calc_fdmt_inputs(float* x, int rows, int cols, float* norm_input, float* stats) {
    float* rmean = stats;
    float* rdisp = stats + rows;
    double sm = 0, s2 = 0, dsum = 0, dsq = 0;
    for (int r = 0; r < rows; ++r) {
        const float* v = x + (size_t)r * cols;
        double s = 0, q = 0;
        for (int t = 0; t < cols; ++t) { s += v[t]; q += (double)v[t] * v[t]; }
        double m = s / cols, d = q / cols - m * m;
        rmean[r] = (float)m;
        rdisp[r] = (float)d;
    }
    /* global moments from the stored float row values, as the reference does */
    for (int r = 0; r < rows; ++r) {
        double m = rmean[r], d = rdisp[r];
        sm += m; s2 += d + m * m;
        dsum += d; dsq += d * d;
    }
    double mean = sm / rows, var = s2 / rows - mean * mean;
    double dmean = dsum / rows, dvar = dsq / rows - dmean * dmean;
    float mf = (float)mean, sf = (float)sqrt(var > 0 ? var : 0);
    float dmf = (float)dmean, dsf = (float)sqrt(dvar > 0 ? dvar : 0);
    stats[2 * rows + 0] = mf; stats[2 * rows + 1] = sf;
    stats[2 * rows + 2] = dmf; stats[2 * rows + 3] = dsf;
    for (int r = 0; r < rows; ++r) {
        float* v = x + (size_t)r * cols;
        float* m = norm_input + (size_t)r * cols;
        if ((double)fabsf(rdisp[r] - dmf) > 4.0 * (double)dsf) {
            for (int t = 0; t < cols; ++t) { v[t] = 0.0f; m[t] = 0.0f; }
        } else {
            for (int t = 0; t < cols; ++t) { v[t] = (v[t] - mf) / sf; m[t] = 1.0f; }
        }
    }
}
