// Search stage on sm_100a: per-row statistics, per-row normalisation and the
// fused normalise + boxcar + candidate-compaction kernel.
//
// Boxcar semantics (reference L/Clusterization/Clusterization.cu):
//   POW2 mode  gather_candidates_in_dynamicalArray_kernel (:420-455): for each
//              start sample t a running sum x[t] + x[t+1] + ... is tested at
//              w = 1, 2, 4, .., 2^Q; mwidth = log2 w;
//   ALL mode   do_plan_kernel / gather_candidates_in_heap_kernel (:592-671):
//              every w = 1..W, mwidth = w (the same running sum, since the
//              reference re-adds x[t..t+w-1] from x[t] in order);
//   a window is only tested when it lies inside the row; S/N = sum / sqrtf(w)
//   and a candidate is emitted when S/N > thr.
// The running sum is sequential from the start sample, as in the reference
// (a prefix-sum difference rounds differently and would flip candidates at
// the threshold).
//
// Compaction: lanes that pass a test are appended with one atomicAdd per warp
// (ballot + popc); the set of candidates is deterministic, their order is not,
// so the list is then sorted by the canonical key (mdt, mt, width) — the
// reference's heap order — with a stable device radix sort.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <cmath>

#include "internal.h"
#include "search_common.cuh"

#define BFS_TRY_ST(x) do { bfs_status st_ = (x); if (st_ != BFS_OK) return st_; } while (0)

namespace bfs {
namespace {

constexpr int kBoxThreads = 256;
constexpr int kBoxTile = 1024;  // start samples per CTA
constexpr int kMaxPow2Q = 16;
constexpr int kMaxAllW = 4096;

// stats[r] = mean, stats[rows + r] = std (mode 0) or population variance (mode 1)
// launched with clusters of gridDim.x CTAs (one cluster per row)
__global__ void __launch_bounds__(kStatThreads)
k_row_stats(const float* __restrict__ plane, int rows, int cols, float* __restrict__ stats,
            int mode, int vec) {
    const int row = blockIdx.y;
    double s, q;
    cluster_row_moments(plane + static_cast<size_t>(row) * cols, row, cols, vec != 0, s, q);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const double mean = s / cols;
        double var = q / cols - mean * mean;
        if (mode == 0) {
            if (var < 0.0) var = 0.0;
            stats[row] = static_cast<float>(mean);
            stats[rows + row] = static_cast<float>(sqrt(var));
        } else {
            stats[row] = static_cast<float>(mean);
            stats[rows + row] = static_cast<float>(var);
        }
    }
}

__device__ __forceinline__ float norm_sample(float v, float m, float s) {
    return s > 0.0f ? __fdiv_rn(__fsub_rn(v, m), s) : 0.0f;
}

__global__ void k_norm_rows(const float* __restrict__ in, float* __restrict__ out, int rows,
                            int cols, const float* __restrict__ stats) {
    const int row = blockIdx.y;
    const float m = stats[row], s = stats[rows + row];
    const size_t base = static_cast<size_t>(row) * cols;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < cols; t += gridDim.x * blockDim.x)
        out[base + t] = norm_sample(__ldg(in + base + t), m, s);
}

template <int MODE>
__global__ void __launch_bounds__(kBoxThreads)
k_boxcar(const float* __restrict__ plane, int rows, int cols, const float* __restrict__ stats,
         const float* __restrict__ d_thr, float thr_host, int wmax, int snr_fast,
         bfs_cand* __restrict__ out, unsigned capacity, unsigned* __restrict__ d_count,
         int tag, int* __restrict__ tags) {
    extern __shared__ float tile[];
    const int row = blockIdx.y;
    const int t0 = blockIdx.x * kBoxTile;
    const float* x = plane + static_cast<size_t>(row) * cols;
    const int span = kBoxTile + wmax - 1;
    float m = 0.0f, sd = 0.0f;
    if (stats) { m = stats[row]; sd = stats[rows + row]; }
    for (int i = threadIdx.x; i < span; i += kBoxThreads) {
        const int t = t0 + i;
        float v = (t < cols) ? __ldg(x + t) : 0.0f;
        if (stats) v = norm_sample(v, m, sd);
        tile[i] = v;
    }
    __syncthreads();
    const float thr = d_thr ? __ldg(d_thr) : thr_host;
    const int lane = threadIdx.x & 31;
#pragma unroll 1
    for (int k = 0; k < kBoxTile / kBoxThreads; ++k) {
        const int i = threadIdx.x + k * kBoxThreads;
        const int t = t0 + i;
        float sum = 0.0f;
        int next = 1, pw = 0;
#pragma unroll 1
        for (int w = 1; w <= wmax; ++w) {
            const bool inside = (t + w - 1) < cols;
            if (inside) sum = __fadd_rn(sum, tile[i + w - 1]);
            bool test;
            int code;
            if (MODE == 0) {
                test = (w == next);
                code = pw;
                if (test) { next <<= 1; ++pw; }
                if (!test) continue;  // warp-uniform: w and next are the same in every lane
            } else {
                test = true;
                code = w;
            }
            const float rw = __fsqrt_rn(static_cast<float>(w));
            const float snr = snr_fast ? __fdividef(sum, rw) : __fdiv_rn(sum, rw);
            const bool pass = inside && test && (snr > thr);
            const unsigned ballot = __ballot_sync(0xffffffffu, pass);
            if (ballot) {
                const int leader = __ffs(ballot) - 1;
                unsigned base = 0;
                if (lane == leader) base = atomicAdd(d_count, static_cast<unsigned>(__popc(ballot)));
                base = __shfl_sync(0xffffffffu, base, leader);
                if (pass) {
                    const unsigned idx = base + __popc(ballot & ((1u << lane) - 1u));
                    if (idx < capacity) {
                        bfs_cand c;
                        c.mt = t; c.mdt = row; c.mwidth = code; c.msnr = snr;
                        out[idx] = c;
                        if (tags) tags[idx] = tag;
                    }
                }
            }
        }
    }
}

// Widest window of the compile-time width sets (pow2 up to 128, every width
// up to 8) and sqrtf(w) for them, computed on the host (IEEE there too).
constexpr int kRegMaxW = 128;

struct WidthConsts {
    float sq[kRegMaxW + 1];  // sqrtf(w), w = 1..kRegMaxW (index w)
};

// ---- ordered boxcar over row pairs -------------------------------------------
// The register-blocked boxcar for two rows at once, writing the candidates
// of every warp's tile as one block in canonical order.  Each warp owns
// kPairWarpTile consecutive starts of rows 2y and 2y + 1 and stages them
// (with the WMAX - 1 samples after them) interleaved in its own shared
// region: position p holds {row 2y, row 2y + 1} at sample tw + p, so one
// packed add.rn.f32x2 advances the running sums of both rows at one start —
// each half is rounded as one __fadd_rn, so the sums are the reference's
// sequential sums bit for bit.  Per width the warp first asks whether any
// of its sums exceeds the width's lower bound of passing sums (a
// three-input max tree and one vote); only then are exact quotients
// evaluated.  The width loop keeps the passing windows as bits (start j,
// width code c) -> bit 8 j + c, which orders them by (start, width), and
// each one's S/N in a per-lane array indexed like its bit; a warp scan of
// the lanes' counts and one atomicAdd give the warp its block (row 2y's
// candidates, then row 2y + 1's), and each lane writes its windows at their
// positions in the block from the bits.  The warps never wait for one
// another.
// Record (row, warp tile i) = {first index, count} of row `row`'s block in
// warp tile i (index row * ceil(cols / kPairWarpTile) + i), so a scan of
// the counts in record order gives every candidate its canonical position
// (compact_ordered).
constexpr int kPairStarts = 8;                            // starts per lane
constexpr int kPairWarpTile = 32 * kPairStarts;           // starts per warp
constexpr int kPairWarps = 4;
constexpr int kPairThreads = 32 * kPairWarps;
constexpr int kPairTile = kPairWarps * kPairWarpTile;     // starts per CTA

__device__ __forceinline__ unsigned long long pack2(float lo, float hi) {
    unsigned long long d;
    asm("mov.b64 %0, {%1, %2};" : "=l"(d) : "f"(lo), "f"(hi));
    return d;
}
__device__ __forceinline__ void unpack2(unsigned long long v, float& lo, float& hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
// both halves rounded to nearest, each exactly as __fadd_rn
__device__ __forceinline__ unsigned long long add2_rn(unsigned long long a, unsigned long long b) {
    unsigned long long d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ float max3f(float a, float b, float c) {
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

// Shared layout of a warp's staged tile: logical float4 f (positions 2f,
// 2f + 1 of both rows) sits at f + f / 4, one float4 of padding after every
// four, so the eight lanes of a quarter warp — whose windows start 4 float4s
// apart — read eight different bank groups.
__device__ __forceinline__ int pad4(int f) { return f + (f >> 2); }

// The width loop of one lane: kPairStarts starts from tb in both rows (win4
// = the warp's staged tile, f0 = the lane's first logical float4).  pass[r] gets bit 8 j + c
// for every passing window (start j, width code c) of row r, and snr[64 r +
// 8 j + c] its S/N.  edge: some window may leave the row (tested per window).
template <int MODE, int WMAX>
__device__ __forceinline__ void pair_widths(const float4* __restrict__ win4, int f0, int tb, int cols, bool edge,
                                            float thr, float thr_lo, int snr_fast, const WidthConsts& wc,
                                            unsigned long long (&pass)[2], float (&snr)[128]) {
    constexpr int S = kPairStarts;
    constexpr int kPos = S + WMAX - 1;   // positions this lane reads
    constexpr int kVec = (kPos + 1) / 2; // float4s (two positions each)
    constexpr int kAhead = 4;            // window pairs are read this many steps before use
    unsigned long long win[2 * kVec];
    unsigned long long sum[S];
    constexpr int kPre = (S + kAhead + 1) / 2 < kVec ? (S + kAhead + 1) / 2 : kVec;
#pragma unroll
    for (int v = 0; v < kPre; ++v) {
        const float4 q = win4[pad4(f0 + v)];
        win[2 * v] = pack2(q.x, q.y);
        win[2 * v + 1] = pack2(q.z, q.w);
    }
#pragma unroll
    for (int j = 0; j < S; ++j) sum[j] = 0ull;   // +0.0 in both halves
#pragma unroll
    for (int w = 1; w <= WMAX; ++w) {
        // step w reads positions w - 1 .. w + S - 2; the pair starting at
        // position w + S - 2 + kAhead is fetched now, kAhead steps early
        const int pn = w + S - 2 + kAhead;
        if ((pn & 1) == 0 && pn / 2 >= kPre && pn / 2 < kVec) {
            const float4 q = win4[pad4(f0 + pn / 2)];
            win[pn] = pack2(q.x, q.y);
            win[pn + 1] = pack2(q.z, q.w);
        }
#pragma unroll
        for (int j = 0; j < S; ++j) sum[j] = add2_rn(sum[j], win[j + w - 1]);
        if (MODE == 0 && (w & (w - 1)) != 0) continue;
        const float sq = wc.sq[w];
        // RN(sum / sq) > thr needs sum > RN(RN(thr sq) (1 - 1e-5)) for thr > 0
        const float lim = thr_lo > -INFINITY ? __fmul_rn(__fmul_rn(thr, sq), 0.99999f) : -INFINITY;
        float h[2 * S], hm[S];
#pragma unroll
        for (int j = 0; j < S; ++j) {
            unpack2(sum[j], h[2 * j], h[2 * j + 1]);
            hm[j] = fmaxf(h[2 * j], h[2 * j + 1]);   // both rows at start j
        }
        float mx = max3f(hm[0], hm[1], hm[2]);
#pragma unroll
        for (int k = 3; k + 1 < S; k += 2) mx = max3f(mx, hm[k], hm[k + 1]);
        if (S % 2 == 0) mx = fmaxf(mx, hm[S - 1]);
        if (!__any_sync(0xffffffffu, mx > lim)) continue;
        const int code = (MODE == 1) ? w - 1 : 31 - __clz(w);
        // windows inside the row: starts j < inside
        const int inside = edge ? cols - (tb + w - 1) : S;
        // windows over the bound: a bit each (one code path for all of them)
        unsigned over = 0;
#pragma unroll
        for (int k = 0; k < 2 * S; ++k)
            if (h[k] > lim && (k >> 1) < inside) over |= 1u << k;
#pragma unroll 1
        while (over) {
            const int k = __ffs(over) - 1;
            over &= over - 1;
            float sj = h[0];
#pragma unroll
            for (int i = 1; i < 2 * S; ++i)
                if (i == k) sj = h[i];
            const float q = snr_fast ? __fdividef(sj, sq) : __fdiv_rn(sj, sq);
            if (q > thr) {
                const int r = k & 1, bit = 8 * (k >> 1) + code;
                pass[r] |= 1ull << bit;
                snr[64 * r + bit] = q;
            }
        }
    }
}

template <int MODE, int WMAX>
__global__ void __launch_bounds__(kPairThreads, WMAX <= 8 ? 8 : WMAX <= 32 ? 6 : WMAX <= 64 ? 4 : 2)
k_boxcar_pair(const float* __restrict__ plane, int rows, int cols, const float* __restrict__ stats,
              const float* __restrict__ d_thr, float thr_host, float thr_lo_host, int snr_fast, int vec,
              bfs_cand* __restrict__ out, unsigned capacity, unsigned* __restrict__ d_count,
              unsigned* __restrict__ rec_first, unsigned* __restrict__ rec_count, const WidthConsts wc) {
    // staged positions of a warp: every start's windows, a multiple of 4
    constexpr int kSpan = (kPairWarpTile + WMAX - 1 + 3) / 4 * 4;
    constexpr int kF4 = kSpan / 2;                      // logical float4s (kSpan positions x 2 rows)
    __shared__ float4 tile4[kPairWarps][kF4 + kF4 / 4]; // padded (pad4)
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wt = blockIdx.x * kPairWarps + warp;     // warp tile
    const int tw = wt * kPairWarpTile;
    if (tw >= cols) return;                            // warp-uniform; no other warp is waited for
    const int row0 = 2 * static_cast<int>(blockIdx.y);
    const bool has1 = row0 + 1 < rows;
    const float* x0 = plane + static_cast<size_t>(row0) * cols;
    const float* x1 = has1 ? x0 + cols : x0;
    float m0 = 0.0f, s0 = 1.0f, m1 = 0.0f, s1 = 1.0f;
    if (stats) {
        m0 = stats[row0]; s0 = stats[rows + row0];
        if (has1) { m1 = stats[row0 + 1]; s1 = stats[rows + row0 + 1]; }
    }
    auto nz = [&](float v, float m, float s) { return stats ? norm_sample(v, m, s) : v; };
    float4* t4 = tile4[warp];
    float* tile = reinterpret_cast<float*>(t4);        // position p, row r at 4 pad4(p / 2) + 2 (p % 2) + r
    const bool interior = tw + kSpan <= cols;
    if (interior && vec) {
        // 16-byte loads of both rows, every load in flight before the first use
        constexpr int kQ = kSpan / 4;                   // float4s per row
        constexpr int kPer = (kQ + 31) / 32;
        float4 a[kPer], b[kPer];
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            const int q = lane + 32 * k;
            if (k < kPer - 1 || q < kQ) {
                a[k] = __ldg(reinterpret_cast<const float4*>(x0 + tw) + q);
                b[k] = has1 ? __ldg(reinterpret_cast<const float4*>(x1 + tw) + q) : make_float4(0.f, 0.f, 0.f, 0.f);
            }
        }
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            const int q = lane + 32 * k;
            if (k < kPer - 1 || q < kQ) {
                const float b0 = has1 ? nz(b[k].x, m1, s1) : 0.0f, b1 = has1 ? nz(b[k].y, m1, s1) : 0.0f;
                const float b2 = has1 ? nz(b[k].z, m1, s1) : 0.0f, b3 = has1 ? nz(b[k].w, m1, s1) : 0.0f;
                t4[pad4(2 * q)] = make_float4(nz(a[k].x, m0, s0), b0, nz(a[k].y, m0, s0), b1);
                t4[pad4(2 * q + 1)] = make_float4(nz(a[k].z, m0, s0), b2, nz(a[k].w, m0, s0), b3);
            }
        }
    } else if (interior) {
        // 4-byte loads (rows not 16-byte aligned), all in flight first
        constexpr int kPer = (kSpan + 31) / 32;
        float a[kPer], b[kPer];
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            const int p = lane + 32 * k;
            if (k < kPer - 1 || p < kSpan) {
                a[k] = __ldg(x0 + tw + p);
                b[k] = has1 ? __ldg(x1 + tw + p) : 0.0f;
            }
        }
        float2* t2 = reinterpret_cast<float2*>(t4);
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            const int p = lane + 32 * k;
            if (k < kPer - 1 || p < kSpan)
                t2[2 * pad4(p >> 1) + (p & 1)] = make_float2(nz(a[k], m0, s0), has1 ? nz(b[k], m1, s1) : 0.0f);
        }
    } else {
        for (int p = lane; p < kSpan; p += 32) {
            const int t = tw + p;
            const bool in = t < cols;
            const int e = 4 * pad4(p >> 1) + 2 * (p & 1);
            tile[e] = in ? nz(__ldg(x0 + t), m0, s0) : 0.0f;
            tile[e + 1] = (in && has1) ? nz(__ldg(x1 + t), m1, s1) : 0.0f;
        }
    }
    __syncwarp();
    float thr = thr_host, thr_lo = thr_lo_host;
    if (d_thr) {
        thr = __ldg(d_thr);
        thr_lo = thr > 0.0f ? thr * 0.99999f : -INFINITY;
    }
    const int p0 = lane * kPairStarts;
    const int tb = tw + p0;
    const int f0 = p0 / 2;
    unsigned long long pass[2] = {0ull, 0ull};
    float snr[128];   // S/N of the passing windows (indexed like their bits)
    pair_widths<MODE, WMAX>(t4, f0, tb, cols, !interior, thr, thr_lo, snr_fast, wc, pass, snr);
    if (!has1) pass[1] = 0ull;

    // the warp's block: row 0's candidates, then row 1's, lanes in order
    const unsigned c0 = __popcll(pass[0]), c1 = __popcll(pass[1]);
    unsigned i0 = c0, i1 = c1;   // inclusive scans over the lanes
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const unsigned u0 = __shfl_up_sync(0xffffffffu, i0, d), u1 = __shfl_up_sync(0xffffffffu, i1, d);
        if (lane >= d) { i0 += u0; i1 += u1; }
    }
    const unsigned tot0 = __shfl_sync(0xffffffffu, i0, 31), tot1 = __shfl_sync(0xffffffffu, i1, 31);
    unsigned first = 0;
    if (lane == 0) {
        first = (tot0 + tot1) ? atomicAdd(d_count, tot0 + tot1) : 0u;
        const int nwt = (cols + kPairWarpTile - 1) / kPairWarpTile;
        const size_t rec = static_cast<size_t>(row0) * nwt + wt;
        rec_first[rec] = first;
        rec_count[rec] = tot0;
        if (has1) {
            rec_first[rec + nwt] = first + tot0;
            rec_count[rec + nwt] = tot1;
        }
    }
    if (tot0 + tot1 == 0) return;   // warp-uniform
    first = __shfl_sync(0xffffffffu, first, 0);
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        unsigned idx = first + (r ? tot0 + i1 - c1 : i0 - c0);
        unsigned long long m = pass[r];
        while (m) {   // bit order = (start, width) order
            const int bit = __ffsll(static_cast<long long>(m)) - 1;
            m &= m - 1;
            if (idx < capacity) {
                const int code = bit & 7;
                bfs_cand c;
                c.mt = tb + (bit >> 3); c.mdt = row0 + r; c.mwidth = MODE == 1 ? code + 1 : code;
                c.msnr = snr[64 * r + bit];
                out[idx] = c;
            }
            ++idx;
        }
    }
}

// Candidates of records [0, nrec) moved to their canonical positions
// (pos = exclusive scan of the counts); tags[pos..] = the record's beam when
// tags is given (beam b owns records [beam_rec[b], beam_rec[b + 1])).  A warp
// takes 32 consecutive records and copies each non-empty one with all lanes.
__global__ void k_compact_records(const bfs_cand* __restrict__ src, const unsigned* __restrict__ rec_first,
                                  const unsigned* __restrict__ rec_count, const unsigned* __restrict__ rec_pos,
                                  long long nrec, const long long* __restrict__ beam_rec, int nb,
                                  bfs_cand* __restrict__ dst, int* __restrict__ tags) {
    const long long r = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    unsigned n = 0, from = 0, to = 0;
    int beam = 0;
    if (r < nrec) {
        n = rec_count[r];
        if (n) {
            from = rec_first[r];
            to = rec_pos[r];
            if (tags) {   // last beam whose first record is <= r
                int lo = 0, hi = nb - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (beam_rec[mid] <= r) lo = mid; else hi = mid - 1;
                }
                beam = lo;
            }
        }
    }
    unsigned todo = __ballot_sync(0xffffffffu, n != 0);
    while (todo) {
        const int src_lane = __ffs(todo) - 1;
        todo &= todo - 1;
        const unsigned cn = __shfl_sync(0xffffffffu, n, src_lane);
        const unsigned cf = __shfl_sync(0xffffffffu, from, src_lane);
        const unsigned ct = __shfl_sync(0xffffffffu, to, src_lane);
        const int cb = __shfl_sync(0xffffffffu, beam, src_lane);
        for (unsigned i = lane; i < cn; i += 32) {
            dst[ct + i] = src[cf + i];
            if (tags) tags[ct + i] = cb;
        }
    }
}

// Canonical key of a candidate: (row * cols + start) << wbits | width code,
// with the width code 0..Q (pow2 mode) or w-1 (all-widths mode).
__device__ __forceinline__ unsigned long long cand_key(const bfs_cand& v, int cols, int mode, int wbits) {
    const unsigned long long cell = static_cast<unsigned long long>(v.mdt) * cols + v.mt;
    const unsigned long long code = static_cast<unsigned long long>(mode == 0 ? v.mwidth : v.mwidth - 1);
    return (cell << wbits) | code;
}

__global__ void k_cand_keys(const bfs_cand* __restrict__ c, unsigned n, int cols, int mode, int wbits,
                            unsigned long long* __restrict__ keys, unsigned* __restrict__ vals) {
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    keys[i] = cand_key(c[i], cols, mode, wbits);
    vals[i] = i;
}

__global__ void k_gather_cands(const bfs_cand* __restrict__ src, const unsigned* __restrict__ idx,
                               unsigned n, bfs_cand* __restrict__ dst) {
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[idx[i]];
}

// 32-bit variant: the key holds the whole position, the S/N rides along as
// the sort value, and the records are rebuilt from (key, S/N).
__global__ void k_cand_keys32(const bfs_cand* __restrict__ c, unsigned n, int cols, int mode, int wbits,
                              unsigned* __restrict__ keys, unsigned* __restrict__ vals) {
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bfs_cand v = c[i];
    keys[i] = static_cast<unsigned>(cand_key(v, cols, mode, wbits));
    vals[i] = __float_as_uint(v.msnr);
}

__global__ void k_cand_decode32(const unsigned* __restrict__ keys, const unsigned* __restrict__ vals,
                                unsigned n, int cols, int mode, int wbits, bfs_cand* __restrict__ out) {
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned k = keys[i];
    const unsigned cell = wbits ? (k >> wbits) : k;
    const int code = static_cast<int>(k & ((1u << wbits) - 1u));
    bfs_cand c;
    c.mt = static_cast<int>(cell % static_cast<unsigned>(cols));
    c.mdt = static_cast<int>(cell / static_cast<unsigned>(cols));
    c.mwidth = mode == 0 ? code : code + 1;
    c.msnr = __uint_as_float(vals[i]);
    out[i] = c;
}

int bits_for(unsigned long long v) {
    int b = 0;
    while (b < 64 && (v >> b) != 0ull) ++b;
    return b;
}

}  // namespace

// Sorts n candidates of a rows x cols plane into the canonical order in place.
// Scratch comes from the stream-ordered pool allocator.
bfs_status sort_candidates_canonical(bfs_cand* d_c, unsigned n, int rows, int cols, int mode,
                                     int param, cudaStream_t s) {
    if (n < 2) return BFS_OK;
    const int wbits = bits_for(static_cast<unsigned long long>(mode == 0 ? param : param - 1));
    const int cell_bits = bits_for(static_cast<unsigned long long>(rows) * cols - 1);
    const int end_bit = cell_bits + wbits;
    const int th = 256, bl = static_cast<int>((n + th - 1) / th);
    void* cub_tmp = nullptr;
    size_t cub_bytes = 0;
    if (end_bit <= 32) {
        unsigned *k = nullptr, *v = nullptr;
        BFS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, cub_bytes, k, k, v, v,
                                                 static_cast<int>(n), 0, end_bit, s));
        BFS_TRY_ST(stream_alloc(reinterpret_cast<void**>(&k), n * sizeof(unsigned) * 4, s));
        v = k + 2 * static_cast<size_t>(n);
        BFS_TRY_ST(stream_alloc(&cub_tmp, cub_bytes ? cub_bytes : 16, s));
        k_cand_keys32<<<bl, th, 0, s>>>(d_c, n, cols, mode, wbits, k, v);
        BFS_LAUNCH_CHECK("k_cand_keys32");
        BFS_CUDA(cub::DeviceRadixSort::SortPairs(cub_tmp, cub_bytes, k, k + n, v, v + n,
                                                 static_cast<int>(n), 0, end_bit, s));
        k_cand_decode32<<<bl, th, 0, s>>>(k + n, v + n, n, cols, mode, wbits, d_c);
        BFS_LAUNCH_CHECK("k_cand_decode32");
        BFS_CUDA(cudaFreeAsync(k, s));
        BFS_CUDA(cudaFreeAsync(cub_tmp, s));
        return BFS_OK;
    }
    unsigned long long *k_in = nullptr, *k_out = nullptr;
    unsigned *v_in = nullptr, *v_out = nullptr;
    bfs_cand* tmp = nullptr;
    BFS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, cub_bytes, k_in, k_out, v_in, v_out,
                                             static_cast<int>(n), 0, end_bit, s));
    BFS_TRY_ST(stream_alloc(reinterpret_cast<void**>(&k_in), n * sizeof(unsigned long long) * 2, s));
    k_out = k_in + n;
    BFS_TRY_ST(stream_alloc(reinterpret_cast<void**>(&v_in), n * sizeof(unsigned) * 2, s));
    v_out = v_in + n;
    BFS_TRY_ST(stream_alloc(reinterpret_cast<void**>(&tmp), n * sizeof(bfs_cand), s));
    BFS_TRY_ST(stream_alloc(&cub_tmp, cub_bytes ? cub_bytes : 16, s));
    k_cand_keys<<<bl, th, 0, s>>>(d_c, n, cols, mode, wbits, k_in, v_in);
    BFS_LAUNCH_CHECK("k_cand_keys");
    BFS_CUDA(cub::DeviceRadixSort::SortPairs(cub_tmp, cub_bytes, k_in, k_out, v_in, v_out,
                                             static_cast<int>(n), 0, end_bit, s));
    k_gather_cands<<<bl, th, 0, s>>>(d_c, v_out, n, tmp);
    BFS_LAUNCH_CHECK("k_gather_cands");
    BFS_CUDA(cudaMemcpyAsync(d_c, tmp, n * sizeof(bfs_cand), cudaMemcpyDeviceToDevice, s));
    BFS_CUDA(cudaFreeAsync(k_in, s));
    BFS_CUDA(cudaFreeAsync(v_in, s));
    BFS_CUDA(cudaFreeAsync(tmp, s));
    BFS_CUDA(cudaFreeAsync(cub_tmp, s));
    return BFS_OK;
}

namespace {
__global__ void k_tagged_keys(const bfs_cand* __restrict__ c, const int* __restrict__ tags, unsigned n,
                              int row_bits, int col_bits, int mode, int wbits,
                              unsigned long long* __restrict__ keys, unsigned* __restrict__ vals) {
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bfs_cand v = c[i];
    const unsigned long long code = static_cast<unsigned long long>(mode == 0 ? v.mwidth : v.mwidth - 1);
    unsigned long long k = static_cast<unsigned long long>(tags[i]);
    k = (k << row_bits) | static_cast<unsigned long long>(v.mdt);
    k = (k << col_bits) | static_cast<unsigned long long>(v.mt);
    keys[i] = (k << wbits) | code;
    vals[i] = i;
}

__global__ void k_gather_tagged(const bfs_cand* __restrict__ src, const int* __restrict__ tsrc,
                                const unsigned* __restrict__ idx, unsigned n, bfs_cand* __restrict__ dst,
                                int* __restrict__ tdst) {
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) { dst[i] = src[idx[i]]; tdst[i] = tsrc[idx[i]]; }
}
}  // namespace

// Canonical order across beams: (tag, row, sample, width); candidates and
// their tags are permuted together (into dst / tdst).
bfs_status sort_tagged_candidates(const bfs_cand* d_c, const int* d_tags, unsigned n, int max_rows,
                                  int max_cols, int max_tag, int mode, int param, bfs_cand* d_dst,
                                  int* d_tdst, cudaStream_t s) {
    if (n == 0) return BFS_OK;
    const int wbits = bits_for(static_cast<unsigned long long>(mode == 0 ? param : param - 1));
    const int row_bits = bits_for(static_cast<unsigned long long>(max_rows - 1));
    const int col_bits = bits_for(static_cast<unsigned long long>(max_cols - 1));
    const int tag_bits = bits_for(static_cast<unsigned long long>(max_tag));
    const int end_bit = tag_bits + row_bits + col_bits + wbits;
    BFS_ARG(end_bit <= 64, "candidate key needs %d bits", end_bit);
    unsigned long long* k = nullptr;
    unsigned* v = nullptr;
    void* tmp = nullptr;
    size_t tmp_bytes = 0;
    BFS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, k, k, v, v, static_cast<int>(n), 0,
                                             end_bit > 0 ? end_bit : 1, s));
    BFS_TRY_ST(stream_alloc(reinterpret_cast<void**>(&k), sizeof(unsigned long long) * 2 * n, s));
    BFS_TRY_ST(stream_alloc(reinterpret_cast<void**>(&v), sizeof(unsigned) * 2 * n, s));
    BFS_TRY_ST(stream_alloc(&tmp, tmp_bytes, s));
    const int th = 256, bl = static_cast<int>((n + th - 1) / th);
    k_tagged_keys<<<bl, th, 0, s>>>(d_c, d_tags, n, row_bits, col_bits, mode, wbits, k, v);
    BFS_LAUNCH_CHECK("k_tagged_keys");
    BFS_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, k, k + n, v, v + n, static_cast<int>(n), 0,
                                             end_bit > 0 ? end_bit : 1, s));
    k_gather_tagged<<<bl, th, 0, s>>>(d_c, d_tags, v + n, n, d_dst, d_tdst);
    BFS_LAUNCH_CHECK("k_gather_tagged");
    BFS_CUDA(cudaFreeAsync(k, s));
    BFS_CUDA(cudaFreeAsync(v, s));
    BFS_CUDA(cudaFreeAsync(tmp, s));
    return BFS_OK;
}

bfs_status launch_row_stats(const float* d_in, int rows, int cols, float* d_stats, int mode,
                            cudaStream_t s) {
    BFS_ARG(d_in && d_stats, "null argument");
    BFS_ARG(rows >= 1 && cols >= 1, "bad shape %dx%d", rows, cols);
    BFS_ARG(rows <= 65535, "rows > 65535 not supported");
    // CTAs per row: doubled while the grid is under two waves of 256-thread
    // CTAs (8 per SM) and every thread still reads >= 32 samples
    int dev = 0, sms = 0;
    BFS_CUDA(cudaGetDevice(&dev));
    BFS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    int split = 1;
    while (split < kStatMaxCluster && static_cast<long long>(rows) * split < 16LL * sms &&
           cols / (2 * split) >= 32 * kStatThreads)
        split *= 2;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(split, rows);
    cfg.blockDim = dim3(kStatThreads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = split;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const int vec = (reinterpret_cast<uintptr_t>(d_in) & 15) == 0 ? 1 : 0;
    BFS_CUDA(cudaLaunchKernelEx(&cfg, k_row_stats, d_in, rows, cols, d_stats, mode, vec));
    return BFS_OK;
}

bfs_status launch_boxcar(const float* d_plane, int rows, int cols, const float* d_stats,
                         float thr, const float* d_thr, int mode, int param, int snr_fast,
                         bfs_cand* d_out, unsigned capacity, unsigned* d_count, cudaStream_t s,
                         int tag, int* d_tags) {
    BFS_ARG(d_plane && d_count, "null argument");
    BFS_ARG(rows >= 1 && cols >= 1 && rows <= 65535, "bad shape %dx%d", rows, cols);
    BFS_ARG(capacity == 0 || d_out, "d_out is null");
    int wmax;
    if (mode == BFS_WIDTHS_POW2) {
        BFS_ARG(param >= 0 && param <= kMaxPow2Q, "Q must be in [0, %d]", kMaxPow2Q);
        wmax = 1 << param;
    } else if (mode == BFS_WIDTHS_ALL) {
        BFS_ARG(param >= 1 && param <= kMaxAllW, "W must be in [1, %d]", kMaxAllW);
        wmax = param;
    } else {
        return fail(BFS_ERR_ARG, "unknown widths_mode %d", mode);
    }
    dim3 grid((cols + kBoxTile - 1) / kBoxTile, rows);
    const size_t smem = sizeof(float) * (kBoxTile + wmax - 1);
    if (mode == BFS_WIDTHS_POW2) {
        if (smem > 48 * 1024)
            BFS_CUDA(cudaFuncSetAttribute(k_boxcar<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          static_cast<int>(smem)));
        k_boxcar<0><<<grid, kBoxThreads, smem, s>>>(d_plane, rows, cols, d_stats, d_thr, thr, wmax,
                                                    snr_fast, d_out, capacity, d_count, tag, d_tags);
    } else {
        if (smem > 48 * 1024)
            BFS_CUDA(cudaFuncSetAttribute(k_boxcar<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          static_cast<int>(smem)));
        k_boxcar<1><<<grid, kBoxThreads, smem, s>>>(d_plane, rows, cols, d_stats, d_thr, thr, wmax,
                                                    snr_fast, d_out, capacity, d_count, tag, d_tags);
    }
    BFS_LAUNCH_CHECK("k_boxcar");
    return BFS_OK;
}

// Whether launch_boxcar_ordered handles a width set (pow2 up to 128 or every
// width up to 8: at most 8 width codes per start).
bool boxcar_ordered_supported(int mode, int param) {
    if (mode == BFS_WIDTHS_POW2) return param >= 0 && param <= 7;
    if (mode == BFS_WIDTHS_ALL) return param >= 1 && param <= 8;
    return false;
}

long long boxcar_ordered_records(int rows, int cols) {
    return static_cast<long long>(rows) * ((cols + kPairWarpTile - 1) / kPairWarpTile);
}

// The boxcar with canonical per-tile output (k_boxcar_pair): candidates go to
// d_out in blocks, one per (row, warp tile), each in canonical order; records
// rec_first / rec_count (boxcar_ordered_records entries, (row, tile) order)
// locate the blocks for compact_ordered.
bfs_status launch_boxcar_ordered(const float* d_plane, int rows, int cols, const float* d_stats, float thr,
                                 const float* d_thr, int mode, int param, int snr_fast, bfs_cand* d_out,
                                 unsigned capacity, unsigned* d_count, unsigned* rec_first, unsigned* rec_count,
                                 cudaStream_t s) {
    BFS_ARG(d_plane && d_count && rec_first && rec_count, "null argument");
    BFS_ARG(rows >= 1 && cols >= 1, "bad shape %dx%d", rows, cols);
    BFS_ARG((rows + 1) / 2 <= 65535, "rows > 131070 not supported");
    BFS_ARG(capacity == 0 || d_out, "d_out is null");
    BFS_ARG(boxcar_ordered_supported(mode, param), "width set (%d, %d) has no ordered kernel", mode, param);
    const float thr_lo = thr > 0.0f ? thr * 0.99999f : -INFINITY;
    const int vec = (cols % 4 == 0) && (reinterpret_cast<uintptr_t>(d_plane) % 16 == 0);
    WidthConsts wc;
    for (int w = 0; w <= kRegMaxW; ++w) wc.sq[w] = std::sqrt(static_cast<float>(w));  // IEEE-correct on the host
    const dim3 grid((cols + kPairTile - 1) / kPairTile, (rows + 1) / 2);
#define BFS_BOX_PAIR(M, W) k_boxcar_pair<M, W><<<grid, kPairThreads, 0, s>>>(                               \
        d_plane, rows, cols, d_stats, d_thr, thr, thr_lo, snr_fast, vec, d_out, capacity, d_count, rec_first, \
        rec_count, wc)
    if (mode == BFS_WIDTHS_POW2) {
        switch (param) {
            case 0: BFS_BOX_PAIR(0, 1); break;
            case 1: BFS_BOX_PAIR(0, 2); break;
            case 2: BFS_BOX_PAIR(0, 4); break;
            case 3: BFS_BOX_PAIR(0, 8); break;
            case 4: BFS_BOX_PAIR(0, 16); break;
            case 5: BFS_BOX_PAIR(0, 32); break;
            case 6: BFS_BOX_PAIR(0, 64); break;
            default: BFS_BOX_PAIR(0, 128); break;
        }
    } else {
        switch (param) {
            case 1: BFS_BOX_PAIR(1, 1); break;
            case 2: BFS_BOX_PAIR(1, 2); break;
            case 3: BFS_BOX_PAIR(1, 3); break;
            case 4: BFS_BOX_PAIR(1, 4); break;
            case 5: BFS_BOX_PAIR(1, 5); break;
            case 6: BFS_BOX_PAIR(1, 6); break;
            case 7: BFS_BOX_PAIR(1, 7); break;
            default: BFS_BOX_PAIR(1, 8); break;
        }
    }
#undef BFS_BOX_PAIR
    BFS_LAUNCH_CHECK("k_boxcar_pair");
    return BFS_OK;
}

// The candidates of nrec records (blocks in src written by
// launch_boxcar_ordered, every count summing to at most the capacity src was
// written with) in canonical order in dst; tags (optional) = each candidate's
// beam, beam b owning records [beam_rec[b], beam_rec[b + 1]) (beam_rec on the
// device, nb + 1 entries).  Scratch from the stream-ordered pool.
bfs_status compact_ordered(const bfs_cand* src, const unsigned* rec_first, const unsigned* rec_count,
                           long long nrec, const long long* beam_rec, int nb, bfs_cand* dst, int* tags,
                           cudaStream_t s) {
    if (nrec <= 0) return BFS_OK;
    BFS_ARG(nrec < (1ll << 31), "too many boxcar tiles (%lld)", nrec);
    BFS_ARG(!tags || (beam_rec && nb >= 1), "tags need the beams' record offsets");
    const int th = 256;
    const long long blocks = (nrec + th - 1) / th;
    BFS_ARG(blocks < (1ll << 31), "too many boxcar tiles (%lld)", nrec);
    unsigned* pos = nullptr;
    void* tmp = nullptr;
    size_t tmp_bytes = 0;
    BFS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, rec_count, pos, static_cast<int>(nrec), s));
    bfs_status st = stream_alloc(reinterpret_cast<void**>(&pos), sizeof(unsigned) * nrec, s);
    if (st == BFS_OK) st = stream_alloc(&tmp, tmp_bytes ? tmp_bytes : 16, s);
    if (st == BFS_OK) {
        cudaError_t e = cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, rec_count, pos, static_cast<int>(nrec), s);
        if (e == cudaSuccess) {
            k_compact_records<<<static_cast<unsigned>(blocks), th, 0, s>>>(src, rec_first, rec_count, pos, nrec,
                                                                            beam_rec, nb, dst, tags);
            e = cudaGetLastError();
        }
        if (e != cudaSuccess) st = fail(BFS_ERR_CUDA, "candidate compaction: %s", cudaGetErrorString(e));
    }
    if (pos) cudaFreeAsync(pos, s);
    if (tmp) cudaFreeAsync(tmp, s);
    return st;
}

}  // namespace bfs

using namespace bfs;

extern "C" bfs_status bfs_row_stats(const float* d_in, int rows, int cols, float* d_stats,
                                    void* stream) {
    return launch_row_stats(d_in, rows, cols, d_stats, 0, as_stream(stream));
}

extern "C" bfs_status bfs_norm_rows(const float* d_in, float* d_out, int rows, int cols,
                                    float* d_stats, void* stream) {
    BFS_ARG(d_in && d_out, "null argument");
    BFS_ARG(rows >= 1 && cols >= 1 && rows <= 65535, "bad shape %dx%d", rows, cols);
    cudaStream_t s = as_stream(stream);
    float* stats = d_stats;
    if (!stats) BFS_TRY_ST(stream_alloc(reinterpret_cast<void**>(&stats), sizeof(float) * 2 * rows, s));
    bfs_status st = launch_row_stats(d_in, rows, cols, stats, 0, s);
    if (st == BFS_OK) {
        dim3 grid(std::min((cols + 255) / 256, 64), rows);
        k_norm_rows<<<grid, 256, 0, s>>>(d_in, d_out, rows, cols, stats);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) st = fail(BFS_ERR_CUDA, "k_norm_rows: %s", cudaGetErrorString(e));
    }
    if (!d_stats) cudaFreeAsync(stats, s);
    return st;
}

extern "C" bfs_status bfs_boxcar_gather(const float* d_plane, int rows, int cols,
                                        const float* d_stats, float thr, const float* d_thr,
                                        int widths_mode, int param, int snr_fast, bfs_cand* d_out,
                                        uint32_t capacity, uint32_t* h_count, void* stream) {
    BFS_ARG(h_count != nullptr, "h_count is null");
    BFS_ARG(d_plane != nullptr, "null argument");
    BFS_ARG(rows >= 1 && cols >= 1 && rows <= 65535, "bad shape %dx%d", rows, cols);
    cudaStream_t s = as_stream(stream);
    // width sets with an ordered kernel: candidates come out in per-tile
    // canonical blocks, then one scan + move puts them in canonical order;
    // others: atomic appends, then a radix sort by the canonical key
    const bool ordered = boxcar_ordered_supported(widths_mode, param);
    const long long nrec = ordered ? boxcar_ordered_records(rows, cols) : 0;
    unsigned* d_count = nullptr;
    unsigned* rec = nullptr;   // first[nrec], count[nrec]
    BFS_TRY_ST(stream_alloc(reinterpret_cast<void**>(&d_count), sizeof(unsigned), s));
    bfs_status st = ordered ? stream_alloc(reinterpret_cast<void**>(&rec), sizeof(unsigned) * 2 * nrec, s) : BFS_OK;
    if (st == BFS_OK) {
        cudaError_t e = cudaMemsetAsync(d_count, 0, sizeof(unsigned), s);
        if (e != cudaSuccess) st = fail(BFS_ERR_CUDA, "cudaMemsetAsync: %s", cudaGetErrorString(e));
    }
    if (st == BFS_OK)
        st = ordered ? launch_boxcar_ordered(d_plane, rows, cols, d_stats, thr, d_thr, widths_mode, param, snr_fast,
                                             d_out, capacity, d_count, rec, rec + nrec, s)
                     : launch_boxcar(d_plane, rows, cols, d_stats, thr, d_thr, widths_mode, param,
                                     snr_fast, d_out, capacity, d_count, s, 0, nullptr);
    unsigned count = 0;
    if (st == BFS_OK) {
        cudaError_t e = cudaMemcpyAsync(&count, d_count, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) st = fail(BFS_ERR_CUDA, "reading the candidate count: %s",
                                        cudaGetErrorString(e));
    }
    cudaFreeAsync(d_count, s);
    if (st == BFS_OK) {
        *h_count = count;
        const unsigned n = count < capacity ? count : capacity;
        if (ordered && count <= capacity && count >= 2) {
            bfs_cand* tmp = nullptr;
            st = stream_alloc(reinterpret_cast<void**>(&tmp), sizeof(bfs_cand) * count, s);
            if (st == BFS_OK) st = compact_ordered(d_out, rec, rec + nrec, nrec, nullptr, 0, tmp, nullptr, s);
            if (st == BFS_OK) {
                cudaError_t e = cudaMemcpyAsync(d_out, tmp, sizeof(bfs_cand) * count, cudaMemcpyDeviceToDevice, s);
                if (e != cudaSuccess) st = fail(BFS_ERR_CUDA, "cudaMemcpyAsync: %s", cudaGetErrorString(e));
            }
            if (tmp) cudaFreeAsync(tmp, s);
        } else if (!ordered || count > capacity) {
            // (ordered overflow: the blocks that fit, sorted)
            st = sort_candidates_canonical(d_out, n, rows, cols, widths_mode, param, s);
        }
    }
    if (rec) cudaFreeAsync(rec, s);
    if (st != BFS_OK) return st;
    if (count > capacity)
        return fail(BFS_ERR_OVERFLOW, "%u candidates found, capacity %u", count, capacity);
    return BFS_OK;
}
