// FDMT plan builder (host).
//
// Restates the reference's plan so the device tables index exactly the rows
// the reference reads:
//   sub-band delay rows   CFdmtB::calc_deltaT            L/FDMT/FdmtB.cpp:201-204
//   level-to-level state  CFdmtB::calcNextStateConfig    L/FDMT/FdmtB.cpp:206-227
//   row cumsums           CFdmtB::calcCumSum_            L/FDMT/FdmtB.cpp:238-245
//   level-0 set-up        CFdmtCpu::create_config        L/FDMT/FdmtCpu.cpp:143-194
//   merge coefficients    CFdmtCpu::fncFdmtIterationC    L/FDMT/FdmtCpu.cpp:286-296
//                         and fnc_delay_h                L/FDMT/FdmtCpu.cpp:369-372
// The arithmetic keeps the reference's types: band edges are float, squared in
// float, reciprocals and differences in double, the merge coefficients are
// float quotients of float delays and the row offsets are float products
// truncated to int.  This file must be compiled with -ffp-contract=off so no
// multiply-add is fused.  The reference GPU class computes the same offsets on
// the device from float reciprocals (fdividef(1.0f, f*f), L/FDMT/FdmtGpu.cu:
// 372-373,466-469) where the CPU class (the parity oracle) takes double
// reciprocals; the CPU class's values are what is reproduced here, once, on
// the host.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "internal.h"

namespace bfs {
namespace {

struct DeltaT {
    float fmin, fmax;
    int max_dt;
    int operator()(float f0, float f1) const {
        const float f0sq = f0 * f0, f1sq = f1 * f1;
        const float lo = fmin * fmin, hi = fmax * fmax;
        const double span = 1.0 / static_cast<double>(f0sq) - 1.0 / static_cast<double>(f1sq);
        const double full = 1.0 / static_cast<double>(lo) - 1.0 / static_cast<double>(hi);
        return static_cast<int>(std::ceil(span / full * (static_cast<double>(max_dt) - 1.0)));
    }
};

// Dispersion delay factor between two band edges, rounded to float.
float edge_delay(float flo, float fhi) {
    const float a = flo * flo, b = fhi * fhi;
    return static_cast<float>(1.0 / static_cast<double>(a) - 1.0 / static_cast<double>(b));
}

}  // namespace

bfs_status build_fdmt_plan(float fmin, float fmax, int nchan, int ncols, int max_dt,
                           FdmtPlanHost* out) {
    BFS_ARG(out != nullptr, "plan output is null");
    BFS_ARG(nchan >= 2, "nchan must be >= 2 (got %d)", nchan);
    BFS_ARG(ncols >= 1, "ncols must be >= 1 (got %d)", ncols);
    BFS_ARG(max_dt >= 1, "max_dt must be >= 1 (got %d)", max_dt);
    BFS_ARG(std::isfinite(fmin) && std::isfinite(fmax) && fmin > 0.0f && fmax > fmin,
            "need 0 < fmin < fmax (got %g, %g)", fmin, fmax);

    FdmtPlanHost& p = *out;
    p = FdmtPlanHost{};
    p.fmin = fmin; p.fmax = fmax; p.nchan = nchan; p.ncols = ncols; p.max_dt = max_dt;
    const DeltaT delta{fmin, fmax, max_dt};

    int q = nchan, n = 0;
    while (q > 1) { q = (q & 1) ? q / 2 + 1 : q / 2; ++n; }
    p.niter = n;
    p.lv.resize(n + 1);

    // level 0
    {
        FdmtLevel& L = p.lv[0];
        const float bw = fmax - fmin;
        const int d0 = delta(fmin, fmin + bw / static_cast<float>(nchan));
        BFS_ARG(d0 >= 0, "negative level-0 delay span");
        p.rows_per_chan0 = d0 + 1;
        L.nsub = nchan;
        L.rows.assign(nchan, d0 + 1);
        L.freq.resize(nchan + 1);
        for (int i = 0; i < nchan; ++i) {
            const float v = static_cast<float>(i) * bw;
            L.freq[i] = fmin + v / static_cast<float>(nchan);
        }
        L.freq[nchan] = fmax;
    }
    // levels 1..n: sub-band bookkeeping
    for (int l = 1; l <= n; ++l) {
        const FdmtLevel& P = p.lv[l - 1];
        FdmtLevel& L = p.lv[l];
        const int qin = P.nsub, half = qin / 2;
        const int qout = (qin & 1) ? half + 1 : half;
        L.nsub = qout;
        L.rows.resize(qout);
        L.freq.resize(qout + 1);
        for (int i = 0; i < half; ++i) {
            L.rows[i] = delta(P.freq[2 * i], P.freq[2 * i + 2]) + 1;
            L.freq[i] = P.freq[2 * i];
        }
        if (qin & 1) {
            L.freq[qout - 1] = P.freq[qin - 1];
            L.rows[qout - 1] = P.rows[qin - 1];
        }
        L.freq[qout] = fmax;
    }
    for (auto& L : p.lv) {
        L.cum.assign(L.nsub + 1, 0);
        for (int i = 0; i < L.nsub; ++i) L.cum[i + 1] = L.cum[i] + L.rows[i];
    }
    BFS_ARG(p.lv[n].total_rows() == max_dt,
            "plan's last level has %d rows, expected max_dt=%d", p.lv[n].total_rows(), max_dt);

    // level 0 look-back: row r of a channel averages x[t-r..t]
    {
        FdmtLevel& L = p.lv[0];
        L.lookback.resize(L.total_rows());
        for (int c = 0; c < nchan; ++c)
            for (int r = 0; r < p.rows_per_chan0; ++r) L.lookback[c * p.rows_per_chan0 + r] = r;
    }
    // merge tables
    for (int l = 1; l <= n; ++l) {
        const FdmtLevel& P = p.lv[l - 1];
        FdmtLevel& L = p.lv[l];
        const int R = L.total_rows(), Rin = P.total_rows();
        L.a_row.resize(R); L.b_row.resize(R); L.shift.resize(R); L.lookback.resize(R);
        for (int i = 0; i < L.nsub; ++i) {
            const int r0 = L.cum[i], nr = L.rows[i];
            if (2 * i + 1 >= P.nsub) {  // odd sub-band count: last one carried over
                for (int j = 0; j < nr; ++j) {
                    L.a_row[r0 + j] = P.cum[2 * i] + j;
                    L.b_row[r0 + j] = -1;
                    L.shift[r0 + j] = 0;
                }
                continue;
            }
            const float all = edge_delay(P.freq[2 * i], P.freq[2 * i + 2]);
            const float c0 = edge_delay(P.freq[2 * i], P.freq[2 * i + 1]) / all;
            const float c1 = edge_delay(P.freq[2 * i + 1], P.freq[2 * i + 2]) / all;
            for (int j = 0; j < nr; ++j) {
                const float fj = static_cast<float>(j);
                const int j0 = static_cast<int>(c0 * fj);
                const int j1 = static_cast<int>(c1 * fj);
                L.a_row[r0 + j] = P.cum[2 * i] + j0;
                L.b_row[r0 + j] = P.cum[2 * i + 1] + j1;
                L.shift[r0 + j] = j0;
            }
        }
        for (int g = 0; g < R; ++g) {
            // The reference indexes the previous plane without bounds checks; a
            // row outside it would be undefined behaviour there, so reject it.
            BFS_ARG(L.a_row[g] >= 0 && L.a_row[g] < Rin && L.b_row[g] < Rin && L.shift[g] >= 0,
                    "level %d row %d references a row outside the previous plane", l, g);
            int lb = P.lookback[L.a_row[g]];
            if (L.b_row[g] >= 0) {
                const int hb = L.shift[g] + P.lookback[L.b_row[g]];
                if (hb > lb) lb = hb;
            }
            L.lookback[g] = lb;
        }
    }
    return BFS_OK;
}

bool build_head_plan(const FdmtPlanHost& p, int k, int tile, size_t smem_limit, HeadPlan* out) {
    if (k < 1 || k > kHeadMaxDepth || k > p.niter || tile < 32) return false;
    const int G = 1 << k;
    if (p.nchan % G != 0) return false;  // every level <= k must pair sub-bands evenly
    for (int l = 1; l <= k; ++l)
        if (p.lv[l].nsub * (1 << l) != p.nchan) return false;
    HeadPlan h;
    h.depth = k;
    h.group = G;
    h.tile = tile;
    const int ngroups = p.nchan / G;
    int max_halo = 0;
    for (int g = 0; g < ngroups; ++g) {
        HeadGroup hg{};
        hg.rows[0] = G * p.rows_per_chan0;
        int rows_a = hg.rows[0], rows_b = 0;
        for (int l = 1; l <= k; ++l) {
            const FdmtLevel& L = p.lv[l];
            const FdmtLevel& P = p.lv[l - 1];
            const int sub_per_group = G >> l;        // sub-bands of this group at level l
            const int s0 = g * sub_per_group;
            const int row0 = L.cum[s0], row1 = L.cum[s0 + sub_per_group];
            const int in0 = P.cum[g * (sub_per_group * 2)];
            hg.rows[l] = row1 - row0;
            hg.tab_off[l] = static_cast<int>(h.tab.size() / 4);
            for (int r = row0; r < row1; ++r) {
                if (L.b_row[r] < 0) return false;    // no carried-over rows inside a group
                h.tab.push_back(L.a_row[r] - in0);
                h.tab.push_back(L.b_row[r] - in0);
                h.tab.push_back(L.shift[r]);
                h.tab.push_back(0);
            }
            if (l < k) {
                if (l & 1) rows_b = std::max(rows_b, hg.rows[l]);
                else rows_a = std::max(rows_a, hg.rows[l]);
            } else {
                hg.out_row0 = row0;
                int lb = 0;
                for (int r = row0; r < row1; ++r) lb = std::max(lb, L.lookback[r]);
                hg.halo = lb;
            }
        }
        h.rows_a = std::max(h.rows_a, rows_a);
        h.rows_b = std::max(h.rows_b, std::max(rows_b, G));  // B also stages the G input rows
        int trows = 0;
        for (int l = 1; l <= k; ++l) trows += hg.rows[l];
        h.tab_rows = std::max(h.tab_rows, trows);
        max_halo = std::max(max_halo, hg.halo);
        h.groups.push_back(hg);
    }
    h.width = ((tile + max_halo) + 31) / 32 * 32;
    if (h.width > 1024) return false;
    h.smem_bytes = static_cast<size_t>(h.rows_a + h.rows_b) * h.width * sizeof(float) +
                   static_cast<size_t>(h.tab_rows) * 4 * sizeof(int);
    if (h.smem_bytes > smem_limit) return false;
    *out = std::move(h);
    return true;
}

bool build_seg_plan(const FdmtPlanHost& p, int l0, int l1, int G, int TT, size_t smem_limit,
                    SegPlan* out, bool from_input, bool single) {
    const int m = l1 - l0;
    if (m < 1 || m > kSegMaxLevels || l0 < 0 || l1 > p.niter || G < 1 || TT != kSegTile) return false;
    const int r0c = p.rows_per_chan0;
    if (from_input && (p.kind != BFS_PLAN_KEITH || l0 != 0 || m < 2 || r0c < 1 || r0c > 5)) return false;
    // window of a row: {lo, hi} = least and largest total head shift from the tile's rows
    struct Win { int row, lo, hi; };
    const int R = p.lv[l1].total_rows();
    std::vector<std::vector<std::vector<Win>>> tiles;  // [tile][i = 0..m] rows sorted by row
    int spread = 0;
    for (int g0 = 0; g0 < R; g0 += G) {
        std::vector<std::vector<Win>> need(m + 1);
        for (int g = g0; g < std::min(R, g0 + G); ++g) need[m].push_back({g, 0, 0});
        for (int i = m; i >= 1; --i) {
            const FdmtLevel& L = p.lv[l0 + i];
            std::vector<Win> below;
            below.reserve(2 * need[i].size());
            for (const Win& w : need[i]) {
                below.push_back({L.a_row[w.row], w.lo, w.hi});
                if (L.b_row[w.row] >= 0)
                    below.push_back({L.b_row[w.row], w.lo + L.shift[w.row], w.hi + L.shift[w.row]});
            }
            std::sort(below.begin(), below.end(), [](const Win& a, const Win& b) { return a.row < b.row; });
            for (const Win& w : below) {
                if (!need[i - 1].empty() && need[i - 1].back().row == w.row) {
                    Win& v = need[i - 1].back();
                    v.lo = std::min(v.lo, w.lo);
                    v.hi = std::max(v.hi, w.hi);
                } else {
                    need[i - 1].push_back(w);
                }
            }
            for (const Win& w : need[i - 1]) spread = std::max(spread, w.hi - w.lo);
        }
        if (from_input) {
            // level-0 row (c, r) at sample t is the running mean of channel c
            // over x[t-r .. t]: the channel's window reaches r samples further
            // left than the row's.  The tile's channels go in front (its
            // input rows); the level-0 rows become a level formed in shared
            // memory.
            std::vector<Win> ch;
            for (const Win& w : need[0]) {
                const int c = w.row / r0c, r = w.row % r0c;
                if (!ch.empty() && ch.back().row == c) {
                    ch.back().lo = std::min(ch.back().lo, w.lo);
                    ch.back().hi = std::max(ch.back().hi, w.hi + r);
                } else {
                    ch.push_back({c, w.lo, w.hi + r});
                }
            }
            need.insert(need.begin(), std::move(ch));
        }
        // input rows start their window on a multiple of 4 samples (16-byte
        // copies): the lead grows to the next multiple of 4, the window by as much
        for (Win& w : need[0]) {
            const int e4 = (w.hi + 3) & ~3;
            spread = std::max(spread, e4 - w.lo);
            w.hi = e4;
        }
        tiles.push_back(std::move(need));
    }
    SegPlan s;
    s.l0 = l0; s.l1 = l1; s.rows = G; s.tile = TT;
    s.r0c = from_input ? r0c : 0;
    // chunks per shared row, rounded up to a count the kernel instantiates
    // (9, 10 or 12 for the 256-sample tile)
    const int nc = (TT + spread + 31) / 32;
    s.nc = nc <= 9 ? 9 : nc <= 10 ? 10 : 12;
    if (nc > kSegMaxChunks) return false;
    s.pitch = 32 * s.nc;
    const int mk = m + (from_input ? 1 : 0);  // levels the kernel forms above its input rows
    if (mk > kSegMaxLevels) return false;
    for (const auto& need : tiles) {
        for (int i = 0; i < mk; ++i) {
            int& r = (i & 1) ? s.rows_y : s.rows_x;
            r = std::max(r, static_cast<int>(need[i].size()));
        }
        s.max_in_rows = std::max(s.max_in_rows, static_cast<int>(need[0].size()));
        s.in_rows += static_cast<int64_t>(need[0].size());
    }
    s.size_x = (s.rows_x + 2) * s.pitch;
    s.size_y = (s.rows_y + 2) * s.pitch;
    s.y0 = s.size_x;
    s.single = single;
    s.x1 = single ? 0 : s.size_x + s.size_y;  // single: X1 is X0
    s.ent_base = single ? s.size_x + s.size_y : s.x1 + s.size_x;
    for (const auto& need : tiles) {
        int ne = 0;
        for (int i = 0; i <= mk; ++i) ne += static_cast<int>(need[i].size());
        s.max_ent = std::max(s.max_ent, ne);
    }
    // entries: one buffer (single), else three (tile j's, j+1's, and j+2's
    // arriving two tiles ahead of use)
    s.smem_bytes = static_cast<size_t>(s.ent_base) * sizeof(float) +
                   (single ? 1 : 3) * static_cast<size_t>(s.max_ent) * 16;
    if (s.smem_bytes > smem_limit) return false;
    auto zero_of = [&](int i) { return ((i & 1) ? s.rows_y : s.rows_x) * s.pitch; };
    auto slot_of = [](const std::vector<Win>& v, int row) {
        auto it = std::lower_bound(v.begin(), v.end(), row, [](const Win& w, int r) { return w.row < r; });
        return static_cast<int>(it - v.begin());
    };
    for (const auto& need : tiles) {
        SegTile st{};
        st.ent = static_cast<int>(s.ent.size() / 4);
        for (int i = 0; i <= mk; ++i) st.n[i] = static_cast<int>(need[i].size());
        for (int j = 0; j < st.n[0]; ++j) {
            const Win& w = need[0][j];
            s.ent.insert(s.ent.end(), {w.row, w.hi, 0, j * s.pitch});
        }
        if (from_input) {
            // level 0 from the channels: x = the channel's sample t, z = the
            // first sample that is not 0 (the row number r, plus the lead),
            // w = destination | r << 20
            for (int j = 0; j < st.n[1]; ++j) {
                const Win& w = need[1][j];
                const int c = w.row / r0c, r = w.row % r0c;
                const int jc = slot_of(need[0], c);
                const int off = need[0][jc].hi - w.hi;
                if (off < r || off > s.pitch || need[0][jc].lo > w.lo) return false;
                s.max_thr = std::max(s.max_thr, r + w.hi);
                if (j * s.pitch >= (1 << 20)) return false;
                s.ent.insert(s.ent.end(), {jc * s.pitch + off, 0, r + w.hi, j * s.pitch | (r << 20)});
            }
        }
        const int k0 = from_input ? 1 : 0;  // need[k0] holds level l0
        for (int i = 1; i <= m; ++i) {
            const FdmtLevel& L = p.lv[l0 + i];
            const std::vector<Win>& lower = need[k0 + i - 1];
            const int ki = k0 + i;                 // kernel level: buffer X when even, Y when odd
            for (int j = 0; j < st.n[ki]; ++j) {
                const Win& w = need[ki][j];
                const int eg = i == m ? 0 : w.hi;  // output rows: lead 0 (samples t0 ..)
                const int ja = slot_of(lower, L.a_row[w.row]);
                const int offa = ja * s.pitch + (lower[ja].hi - eg);
                int offb = zero_of(ki - 1), thr = 0;
                if (L.b_row[w.row] >= 0) {
                    const int jb = slot_of(lower, L.b_row[w.row]);
                    const int sh = L.shift[w.row];
                    offb = jb * s.pitch + (lower[jb].hi - eg - sh);
                    thr = sh + eg;
                    s.max_thr = std::max(s.max_thr, thr);
                    // the head row's window covers every sample this row reads
                    if (lower[jb].hi - eg - sh < 0 || lower[jb].lo > w.lo + sh) return false;
                    if (lower[jb].hi - eg - sh > s.pitch) return false;
                }
                if (lower[ja].hi - eg < 0 || lower[ja].lo > w.lo || lower[ja].hi - eg > s.pitch) return false;
                const int dst = i == m ? w.row : j * s.pitch;
                s.ent.insert(s.ent.end(), {offa, offb, thr, dst});
            }
        }
        s.tiles.push_back(st);
    }
    *out = std::move(s);
    return true;
}

void build_adjoint_tables(const FdmtPlanHost& p, AdjointTables* out) {
    out->off_pos.assign(p.niter + 1, 0);
    out->ent_pos.assign(p.niter + 1, 0);
    out->off.clear();
    out->ent.clear();
    for (int l = 1; l <= p.niter; ++l) {
        const FdmtLevel& L = p.lv[l];
        const int nin = p.lv[l - 1].total_rows();
        const int nout = L.total_rows();
        std::vector<int> cnt(nin + 1, 0);
        for (int g = 0; g < nout; ++g) {
            ++cnt[L.a_row[g] + 1];
            if (L.b_row[g] >= 0) ++cnt[L.b_row[g] + 1];
        }
        for (int i = 0; i < nin; ++i) cnt[i + 1] += cnt[i];
        out->off_pos[l] = out->off.size();
        out->ent_pos[l] = out->ent.size() / 2;
        out->off.insert(out->off.end(), cnt.begin(), cnt.end());
        std::vector<int> fill(cnt.begin(), cnt.end() - 1);
        std::vector<int> ent(2 * static_cast<size_t>(cnt[nin]));
        for (int g = 0; g < nout; ++g) {  // ascending g: each row's list is in g order
            int k = fill[L.a_row[g]]++;
            ent[2 * k] = g;
            ent[2 * k + 1] = 0;
            if (L.b_row[g] >= 0) {
                k = fill[L.b_row[g]]++;
                ent[2 * k] = g;
                ent[2 * k + 1] = L.shift[g];
            }
        }
        out->ent.insert(out->ent.end(), ent.begin(), ent.end());
    }
    out->built = true;
}

// ---------------------------------------------------------------------------
// Pravir plan.  Restates MyVSLib_C++/FDMT_PRAVIR/fdmt_base.cpp:86-278 with
// fdmtUtils.cpp:36-45,92-108, keeping the reference's float arithmetic: the
// dispersion coefficient of a sub-band is a float quotient of float powers
// (std::pow(float, float)), delays are float products rounded with
// std::round, the nearest grid index prefers the upper neighbour on ties.
// ---------------------------------------------------------------------------
namespace {

float pravir_cff(float f1s, float f1e, float f2s, float f2e) {
    const float e = -2.0f;
    return (std::pow(f1s, e) - std::pow(f1e, e)) / (std::pow(f2s, e) - std::pow(f2e, e));
}

long pravir_round(float v) { return static_cast<long>(std::round(v)); }

std::vector<int> pravir_grid(float fs, float fe, float fmin, float fmax, int dt_max, int dt_min, int step) {
    const float r = pravir_cff(fs, fe, fmin, fmax);
    const long hi = pravir_round(static_cast<float>(dt_max) * r);
    const long lo = pravir_round(static_cast<float>(dt_min) * r);
    std::vector<int> g;
    for (long d = lo; d <= hi; d += step) g.push_back(static_cast<int>(d));
    return g;
}

int pravir_closest(const std::vector<int>& g, long v) {
    const auto it = std::lower_bound(g.begin(), g.end(), v);
    int idx = static_cast<int>(it - g.begin());
    if (it != g.end()) {
        if (it != g.begin() && v - *(it - 1) < *it - v) --idx;
    } else {
        idx = static_cast<int>(g.size()) - 1;
    }
    return idx;
}

}  // namespace

bfs_status build_pravir_plan(float fmin, float fmax, int nchan, int ncols, int dt_max, int dt_step,
                             int dt_min, FdmtPlanHost* out) {
    BFS_ARG(out != nullptr, "plan output is null");
    BFS_ARG(nchan >= 2, "nchan must be >= 2 (got %d)", nchan);
    BFS_ARG(ncols >= 1, "ncols must be >= 1 (got %d)", ncols);
    BFS_ARG(dt_step >= 1 && dt_min >= 0 && dt_max >= dt_min, "need dt_step >= 1, 0 <= dt_min <= dt_max");
    BFS_ARG(std::isfinite(fmin) && std::isfinite(fmax) && fmin > 0.0f && fmax > fmin,
            "need 0 < fmin < fmax (got %g, %g)", fmin, fmax);
    FdmtPlanHost& p = *out;
    p = FdmtPlanHost{};
    p.kind = BFS_PLAN_PRAVIR;
    p.fmin = fmin; p.fmax = fmax; p.nchan = nchan; p.ncols = ncols;
    int n = 0;
    while ((1 << n) < nchan) ++n;
    p.niter = n;
    p.lv.resize(n + 1);
    const float df = (fmax - fmin) / static_cast<float>(nchan);
    const float corr = df / 2;

    // level 0: one sub-band per channel, rows = its delay grid
    std::vector<std::vector<int>> grids(nchan);
    {
        FdmtLevel& L = p.lv[0];
        L.nsub = nchan;
        L.rows.resize(nchan);
        for (int i = 0; i < nchan; ++i) {
            const float fs = df * static_cast<float>(i) + fmin;
            const float fe = fs + df;
            grids[i] = pravir_grid(fs, fe, fmin, fmax, dt_max, dt_min, dt_step);
            BFS_ARG(!grids[i].empty(), "channel %d has an empty delay grid", i);
            L.rows[i] = static_cast<int>(grids[i].size());
            for (int d : grids[i]) p.dt0.push_back(d);
        }
    }
    std::vector<int> top = grids[nchan - 1];
    float df_top = df, df_bot = df;
    for (int l = 1; l <= n; ++l) {
        const FdmtLevel& P = p.lv[l - 1];
        FdmtLevel& L = p.lv[l];
        const int nprev = P.nsub;
        const int ncur = nprev / 2 + nprev % 2;
        const bool do_copy = nprev % 2 == 1;
        const float dtop = do_copy ? df_top : df_top + df_bot;
        const float dbot = df_bot * 2;
        std::vector<std::vector<int>> cur(ncur);
        std::vector<float> fst(ncur), fen(ncur), fmd(ncur);
        for (int i = 0; i < ncur; ++i) {
            const float fs = dbot * static_cast<float>(i) + fmin;
            float fe, fm;
            if (i == ncur - 1) {
                if (do_copy) {
                    fe = fs + dtop * 2;
                    fm = fs + dtop;
                    cur[i] = top;
                } else {
                    fe = fs + dtop;
                    fm = fs + dbot / 2;
                    cur[i] = pravir_grid(fs, fe, fmin, fmax, dt_max, dt_min, dt_step);
                    top = cur[i];
                }
            } else {
                fe = fs + dbot;
                fm = fs + dbot / 2;
                cur[i] = pravir_grid(fs, fe, fmin, fmax, dt_max, dt_min, dt_step);
            }
            BFS_ARG(!cur[i].empty(), "level %d sub-band %d has an empty delay grid", l, i);
            fst[i] = fs; fen[i] = fe; fmd[i] = fm;
        }
        L.nsub = ncur;
        L.rows.resize(ncur);
        for (int i = 0; i < ncur; ++i) L.rows[i] = static_cast<int>(cur[i].size());
        L.cum.assign(ncur + 1, 0);
        for (int i = 0; i < ncur; ++i) L.cum[i + 1] = L.cum[i] + L.rows[i];
        std::vector<int> pcum(nprev + 1, 0);
        for (int i = 0; i < nprev; ++i) pcum[i + 1] = pcum[i] + P.rows[i];
        const int R = L.cum[ncur];
        L.a_row.resize(R); L.b_row.resize(R); L.shift.resize(R); L.lookback.assign(R, 0);
        for (int i = 0; i < ncur; ++i) {
            const int tail = 2 * i, head = 2 * i + 1;
            const float fs = fst[i], fe = fen[i];
            const float fm1 = fmd[i] - corr, fm2 = fmd[i] + corr;
            for (int j = 0; j < L.rows[i]; ++j) {
                const long dt = cur[i][j];
                const long m1 = pravir_round(static_cast<float>(dt) * pravir_cff(fs, fm1, fs, fe));
                const long m2 = pravir_round(static_cast<float>(dt) * pravir_cff(fs, fm2, fs, fe));
                BFS_ARG(m1 <= dt && m2 <= dt, "level %d: mid-band delay above the delay", l);
                const int row = L.cum[i] + j;
                if (i == ncur - 1 && do_copy) {
                    L.a_row[row] = pcum[tail] + pravir_closest(grids[tail], dt);
                    L.b_row[row] = -1;
                    L.shift[row] = 0;
                } else {
                    BFS_ARG(m2 < ncols, "level %d: offset %ld >= ncols %d", l, m2, ncols);
                    L.a_row[row] = pcum[tail] + pravir_closest(grids[tail], m1);
                    L.b_row[row] = pcum[head] + pravir_closest(grids[head], dt - m2);
                    L.shift[row] = static_cast<int>(m2);
                }
            }
        }
        grids = std::move(cur);
        df_top = dtop;
        df_bot = dbot;
    }
    for (auto& L : p.lv) {
        if (L.cum.size() != static_cast<size_t>(L.nsub + 1)) {
            L.cum.assign(L.nsub + 1, 0);
            for (int i = 0; i < L.nsub; ++i) L.cum[i + 1] = L.cum[i] + L.rows[i];
        }
    }
    p.dt_out = grids[0];
    p.max_dt = p.out_rows();
    p.rows_per_chan0 = 0;
    return BFS_OK;
}

void build_ones_delays(const FdmtPlanHost& p, std::vector<int>* tau, int* max_tau) {
    // channel and delay of every level-0 row
    const int r0 = p.lv[0].total_rows();
    std::vector<int> chan(r0), delay(r0);
    for (int c = 0; c < p.nchan; ++c)
        for (int r = p.lv[0].cum[c]; r < p.lv[0].cum[c + 1]; ++r) {
            chan[r] = c;
            delay[r] = p.kind == BFS_PLAN_PRAVIR ? p.dt0[r] : r - p.lv[0].cum[c];
        }
    const int nout = p.out_rows();
    tau->assign(static_cast<size_t>(nout) * p.nchan, 0);
    *max_tau = 0;
    // depth-first walk from every output row down to its level-0 rows
    struct Node { int level, row, acc; };
    std::vector<Node> stack;
    for (int d = 0; d < nout; ++d) {
        int* t = tau->data() + static_cast<size_t>(d) * p.nchan;
        stack.clear();
        stack.push_back({p.niter, d, 0});
        while (!stack.empty()) {
            const Node n = stack.back();
            stack.pop_back();
            if (n.level == 0) {
                const int v = n.acc + delay[n.row];
                t[chan[n.row]] = v;
                *max_tau = std::max(*max_tau, v);
                continue;
            }
            const FdmtLevel& L = p.lv[n.level];
            stack.push_back({n.level - 1, L.a_row[n.row], n.acc});
            if (L.b_row[n.row] >= 0) stack.push_back({n.level - 1, L.b_row[n.row], n.acc + L.shift[n.row]});
        }
    }
}

}  // namespace bfs
