// Adjoint FDMT and adjoint boxcar S/N on sm_100a (no reference counterpart:
// the reference has no gradients).  They make the search differentiable, so
// per-channel weights (bandpass / RFI masks) can be optimised against the
// S/N of detections.
//
// Every FDMT level is linear in its input plane, so the adjoint needs only
// the incoming gradient, never the forward planes: nothing is stored and
// nothing is recomputed beyond one pass per level, in two ping-pong planes
// like the forward.
//
//   merge level l   forward  out[g][t] = in[a_g][t] + [t >= s_g] in[b_g][t - s_g]
//                   adjoint  gin[i][u] = sum over the level-l rows g that read
//                            row i of gout[g][u + s] (s = 0 as tail a_g, s_g as
//                            head b_g; terms with u + s >= ncols vanish) — a
//                            gather over the plan's inverse row tables, summed
//                            in ascending g, so the FP32 result is fixed;
//   level 0         forward  P[c,r][t] = [t >= r] mean(x[c][t-r .. t])
//                   adjoint  gx[c][u] = sum_{r'} RN(1/(r'+1)) *
//                            sum_{r=0..r'} [u+r >= r'][u+r < ncols] g0[c,r'][u+r]
//                            (inner sums r ascending, outer r' ascending).
//
// Boxcar S/N at a cell (row d, start t, width w) of the plane y with row mean
// m_d and standard deviation s_d (population, as bfs_row_stats gives):
//   S = sum_{j<w} z(y[d][t+j]) / sqrt(w),  z(v) = (v - m_d) / s_d,
// evaluated exactly as the boxcar kernels do.  Its gradient, with m_d and s_d
// functions of the row (N = ncols samples):
//   dS/dy[d][u] = ([t <= u < t+w] - w/N) / (s_d sqrt(w)) - S (y[d][u] - m_d) / (N s_d^2).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "fdmt_plan.h"
#include "internal.h"

namespace bfs {
namespace {

constexpr int kAdjThreads = 128;   // measured: 128 > 256 > 512 on 1024 x 65536
constexpr int kAdjVecs = 2;       // float4 column groups per thread
constexpr int kAdjInitThreads = 256;

// words w[0..7] = the 8 floats of vectors (q+sv, q+sv+1); elements R..R+3
template <int R>
__device__ __forceinline__ float4 cut4(const float (&w)[8]) {
    return make_float4(w[R], w[R + 1], w[R + 2], w[R + 3]);
}
__device__ __forceinline__ float4 cut4(const float (&w)[8], int r) {
    switch (r) {
        case 1: return cut4<1>(w);
        case 2: return cut4<2>(w);
        default: return cut4<3>(w);
    }
}

// One adjoint merge level: input row i of level l-1 (grid.x) gathers from the
// level-l gradient rows that read it.  VIN: the gradient rows are 16-byte
// aligned with a pitch multiple of 4 (workspace planes, or the caller's plane
// when ncols % 4 == 0): each read moves as the aligned float4 q + sv of this
// thread plus the next one from the neighbouring lane (warp shuffle; lane 31
// loads its own); else as scalars.  The output is a workspace plane (128-byte
// pitch): float4 stores.
// grid: (rows of level l-1, ceil(ceil(ncols / 4) / (256 * kAdjVecs)))
template <bool VIN>
__global__ void __launch_bounds__(kAdjThreads)
k_fdmt_adj_level(const float* __restrict__ gout, float* __restrict__ gin, const int* __restrict__ off,
                 const int2* __restrict__ ent, int ncols, int out_pitch, int in_pitch) {
    const int i = blockIdx.x;
    const int beg = __ldg(off + i), end = __ldg(off + i + 1);
    const int nv = (ncols + 3) >> 2;
    const int lane = threadIdx.x & 31;
    const int base = blockIdx.y * (kAdjThreads * kAdjVecs) + threadIdx.x;
    float acc[kAdjVecs][4];
#pragma unroll
    for (int k = 0; k < kAdjVecs; ++k)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[k][j] = 0.0f;
    for (int e = beg; e < end; ++e) {  // uniform over the block
        const int2 en = __ldg(ent + e);
        const int s = en.y;
        const float* row = gout + static_cast<size_t>(en.x) * out_pitch;
#pragma unroll
        for (int k = 0; k < kAdjVecs; ++k) {
            const int q = base + k * kAdjThreads;
            const int t = 4 * q;
            float v[4];
            if constexpr (VIN) {
                const int sv = s >> 2, r = s & 3;
                const float4* rv = reinterpret_cast<const float4*>(row);
                const int qa = q + sv;
                float4 lo = (qa < nv) ? __ldg(rv + qa) : make_float4(0.f, 0.f, 0.f, 0.f);
                if (r != 0) {
                    float4 hi;
                    hi.x = __shfl_down_sync(0xffffffffu, lo.x, 1);
                    hi.y = __shfl_down_sync(0xffffffffu, lo.y, 1);
                    hi.z = __shfl_down_sync(0xffffffffu, lo.z, 1);
                    hi.w = __shfl_down_sync(0xffffffffu, lo.w, 1);
                    if (lane == 31) hi = (qa + 1 < nv) ? __ldg(rv + qa + 1) : make_float4(0.f, 0.f, 0.f, 0.f);
                    const float w[8] = {lo.x, lo.y, lo.z, lo.w, hi.x, hi.y, hi.z, hi.w};
                    lo = cut4(w, r);
                }
                v[0] = lo.x; v[1] = lo.y; v[2] = lo.z; v[3] = lo.w;
            } else {
#pragma unroll
                for (int j = 0; j < 4; ++j) v[j] = (t + j + s < ncols) ? __ldg(row + t + j + s) : 0.0f;
            }
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (t + j + s < ncols) acc[k][j] = __fadd_rn(acc[k][j], v[j]);
        }
    }
    float* o = gin + static_cast<size_t>(i) * in_pitch;
#pragma unroll
    for (int k = 0; k < kAdjVecs; ++k) {
        const int q = base + k * kAdjThreads;
        if (q < nv) reinterpret_cast<float4*>(o)[q] = make_float4(acc[k][0], acc[k][1], acc[k][2], acc[k][3]);
    }
}

// Adjoint of level 0 (running means), one window sum and one product per
// level-0 row:
//   gx[c][u] = sum_{r'} RN(1/(r'+1)) * sum_{r=0..r'} [u+r >= r'][u+r < ncols] g0[c,r'][u+r]
// (inner sums r ascending, outer r' ascending).  Thread q owns samples
// 4q..4q+3: each row r' is read as the aligned float4 q plus the next one
// from the lane above (warp shuffle; lane 31 loads its own), which covers
// u + r <= 4q + 7 for up to 5 rows per channel (R0C <= 5; R0C = 0: any
// count, scalar reads).  grid: (ceil(ceil(ncols / 4) / 256), nchan)
template <int R0C>
__global__ void __launch_bounds__(kAdjInitThreads)
k_fdmt_adj_init(const float* __restrict__ g0, float* __restrict__ gx, int ncols, int in_pitch,
                int rows_per_chan, int vec_out) {
    const int c = blockIdx.y;
    const float* g = g0 + static_cast<size_t>(c) * rows_per_chan * in_pitch;
    float* o = gx + static_cast<size_t>(c) * ncols;
    const int nv = (ncols + 3) >> 2;
    const int q = blockIdx.x * kAdjInitThreads + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const int u = 4 * q;
    float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    const int R = R0C > 0 ? R0C : rows_per_chan;
    for (int rr = 0; rr < R; ++rr) {
        const float* row = g + static_cast<size_t>(rr) * in_pitch;
        const float rcp = __frcp_rn(static_cast<float>(rr + 1));
        float e[8];
        if constexpr (R0C > 0) {
            const float4 lo = (q < nv) ? __ldg(reinterpret_cast<const float4*>(row) + q)
                                       : make_float4(0.f, 0.f, 0.f, 0.f);
            float4 hi;
            hi.x = __shfl_down_sync(0xffffffffu, lo.x, 1);
            hi.y = __shfl_down_sync(0xffffffffu, lo.y, 1);
            hi.z = __shfl_down_sync(0xffffffffu, lo.z, 1);
            hi.w = __shfl_down_sync(0xffffffffu, lo.w, 1);
            if (lane == 31)
                hi = (q + 1 < nv) ? __ldg(reinterpret_cast<const float4*>(row) + q + 1)
                                  : make_float4(0.f, 0.f, 0.f, 0.f);
            e[0] = lo.x; e[1] = lo.y; e[2] = lo.z; e[3] = lo.w;
            e[4] = hi.x; e[5] = hi.y; e[6] = hi.z; e[7] = hi.w;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            float w = 0.0f;
            const int rmax = R0C > 0 ? R0C : rows_per_chan;
#pragma unroll
            for (int r = 0; r < rmax; ++r) {
                if (r > rr) break;
                const int t = u + j + r;
                if (t >= rr && t < ncols) {
                    float v;
                    if constexpr (R0C > 0) v = e[j + r];
                    else v = __ldg(row + t);
                    w = __fadd_rn(w, v);
                }
            }
            acc[j] = __fadd_rn(acc[j], __fmul_rn(w, rcp));
        }
    }
    if (q >= nv) return;
    if (vec_out && u + 3 < ncols) {
        reinterpret_cast<float4*>(o)[q] = make_float4(acc[0], acc[1], acc[2], acc[3]);
    } else {
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (u + j < ncols) o[u + j] = acc[j];
    }
}

// The last adjoint merge level (level 1 -> level 0) fused with the adjoint of
// level 0 (Keith plans, R0C level-0 rows per channel): for each of channel
// c's level-0 rows the CTA gathers the row's gradient over its samples into
// shared memory (the k_fdmt_adj_level gather of one float4 per thread) and
// folds it into gx at once (the k_fdmt_adj_init sum), so the level-0
// gradient plane is never written or read back.  The sums and their order
// are those of the two kernels, so the bits are too.  CTA b gathers quads
// 255 b .. 255 b + 255 and writes gx for the first 255 of them (each quad's
// window reaches into the next one).  gout: 16-byte aligned rows, pitch a
// multiple of 4.  grid: (ceil(ceil(ncols / 4) / 255), nchan)
template <int R0C>
__global__ void __launch_bounds__(kAdjInitThreads)
k_fdmt_adj_level0(const float* __restrict__ gout, float* __restrict__ gx, const int* __restrict__ off,
                  const int2* __restrict__ ent, int ncols, int out_pitch, int vec_out) {
    constexpr int kOut = kAdjInitThreads - 1;   // quads written per CTA
    __shared__ float4 tile[kAdjInitThreads];
    const int c = blockIdx.y;
    const int nv = (ncols + 3) >> 2;
    const int lane = threadIdx.x & 31;
    const int q = blockIdx.x * kOut + threadIdx.x;
    const int u = 4 * q;
    float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll 1
    for (int rr = 0; rr < R0C; ++rr) {
        const int i = c * R0C + rr;   // level-0 row (c, rr)
        const int beg = __ldg(off + i), end = __ldg(off + i + 1);
        float g[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        for (int e = beg; e < end; ++e) {  // uniform over the block
            const int2 en = __ldg(ent + e);
            const int s = en.y;
            const float4* rv = reinterpret_cast<const float4*>(gout + static_cast<size_t>(en.x) * out_pitch);
            const int sv = s >> 2, r = s & 3;
            const int qa = q + sv;
            float4 lo = (qa < nv) ? __ldg(rv + qa) : make_float4(0.f, 0.f, 0.f, 0.f);
            if (r != 0) {
                float4 hi;
                hi.x = __shfl_down_sync(0xffffffffu, lo.x, 1);
                hi.y = __shfl_down_sync(0xffffffffu, lo.y, 1);
                hi.z = __shfl_down_sync(0xffffffffu, lo.z, 1);
                hi.w = __shfl_down_sync(0xffffffffu, lo.w, 1);
                if (lane == 31) hi = (qa + 1 < nv) ? __ldg(rv + qa + 1) : make_float4(0.f, 0.f, 0.f, 0.f);
                const float w[8] = {lo.x, lo.y, lo.z, lo.w, hi.x, hi.y, hi.z, hi.w};
                lo = cut4(w, r);
            }
            const float v[4] = {lo.x, lo.y, lo.z, lo.w};
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (u + j + s < ncols) g[j] = __fadd_rn(g[j], v[j]);
        }
        tile[threadIdx.x] = make_float4(g[0], g[1], g[2], g[3]);
        __syncthreads();
        if (threadIdx.x < kOut) {
            const float4 a = tile[threadIdx.x], b = tile[threadIdx.x + 1];
            const float e8[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
            const float rcp = __frcp_rn(static_cast<float>(rr + 1));
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                float w = 0.0f;
#pragma unroll
                for (int r = 0; r < R0C; ++r) {
                    if (r > rr) break;
                    const int t = u + j + r;
                    if (t >= rr && t < ncols) w = __fadd_rn(w, e8[j + r]);
                }
                acc[j] = __fadd_rn(acc[j], __fmul_rn(w, rcp));
            }
        }
        __syncthreads();   // the tile is rewritten for the next row
    }
    if (threadIdx.x >= kOut || q >= nv) return;
    float* o = gx + static_cast<size_t>(c) * ncols;
    if (vec_out && u + 3 < ncols) {
        reinterpret_cast<float4*>(o)[q] = make_float4(acc[0], acc[1], acc[2], acc[3]);
    } else {
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (u + j < ncols) o[u + j] = acc[j];
    }
}

// Adjoint of a Pravir plan's level 0 (rows with delays dt_k per channel,
// lvl0 = row cumsum then delays): the same window-mean transpose,
//   gx[c][u] = sum_k RN(1/(dt_k+1)) * sum_{j=0..dt_k} [u+j >= dt_k][u+j < ncols] g0[k][u+j].
// grid: (ceil(ncols / 256), nchan)
__global__ void __launch_bounds__(kAdjInitThreads)
k_fdmt_adj_init_grid(const float* __restrict__ g0, float* __restrict__ gx, const int* __restrict__ lvl0,
                     int nchan, int ncols, int in_pitch) {
    const int c = blockIdx.y;
    const int u = blockIdx.x * kAdjInitThreads + threadIdx.x;
    if (u >= ncols) return;
    const int r0 = __ldg(lvl0 + c), nr = __ldg(lvl0 + c + 1) - r0;
    const int* dts = lvl0 + nchan + 1 + r0;
    float acc = 0.0f;
    for (int k = 0; k < nr; ++k) {
        const int d = __ldg(dts + k);
        const float* row = g0 + static_cast<size_t>(r0 + k) * in_pitch;
        float w = 0.0f;
        for (int j = 0; j <= d; ++j) {
            const int t = u + j;
            if (t >= d && t < ncols) w = __fadd_rn(w, __ldg(row + t));
        }
        acc = __fadd_rn(acc, __fmul_rn(w, __frcp_rn(static_cast<float>(d + 1))));
    }
    gx[static_cast<size_t>(c) * ncols + u] = acc;
}

// S/N at cells: cells[3k..3k+2] = {row, start, width}.  A cell outside the
// plane gives NaN.
__global__ void k_snr_cells(const float* __restrict__ plane, int rows, int cols,
                            const float* __restrict__ stats, const int* __restrict__ cells, int n,
                            float* __restrict__ snr) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int d = cells[3 * k], t = cells[3 * k + 1], w = cells[3 * k + 2];
    if (d < 0 || d >= rows || t < 0 || w < 1 || w > cols - t) { snr[k] = __int_as_float(0x7fc00000); return; }
    const float m = stats[d], sd = stats[rows + d];
    const float* x = plane + static_cast<size_t>(d) * cols + t;
    float sum = 0.0f;
    for (int j = 0; j < w; ++j)
        sum = __fadd_rn(sum, sd > 0.0f ? __fdiv_rn(__fsub_rn(__ldg(x + j), m), sd) : 0.0f);
    snr[k] = __fdiv_rn(sum, __fsqrt_rn(static_cast<float>(w)));
}

// Gradient of sum_k gsnr[k] * S_k with respect to the plane: one CTA per
// row; warp 0 collects the row's cells in cell order (ballot compaction,
// up to kMaxCellsPerRow) and the row constants; then every sample of the
// row is written (rows without cells get zeros).
constexpr int kMaxCellsPerRow = 512;

__global__ void __launch_bounds__(256)
k_snr_cells_adjoint(const float* __restrict__ plane, int rows, int cols, const float* __restrict__ stats,
                    const int* __restrict__ cells, int n, const float* __restrict__ snr,
                    const float* __restrict__ gsnr, float* __restrict__ gplane, int* __restrict__ err) {
    __shared__ int s_t[kMaxCellsPerRow], s_w[kMaxCellsPerRow];
    __shared__ float s_c[kMaxCellsPerRow];  // gsnr / (sd sqrt(w))
    __shared__ int s_n;
    __shared__ float s_a, s_b;              // constant term, coefficient of (y - m)
    const int d = blockIdx.x;
    const float m = stats[d], sd = stats[rows + d];
    const float nf = static_cast<float>(cols);
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        int cnt = 0;
        float a = 0.0f, b = 0.0f;
        for (int k0 = 0; k0 < n; k0 += 32) {
            const int k = k0 + lane;
            const bool mine = k < n && cells[3 * k] == d;
            const unsigned bal = __ballot_sync(0xffffffffu, mine);
            if (mine) {
                const int pos = cnt + __popc(bal & ((1u << lane) - 1u));
                if (pos < kMaxCellsPerRow) {
                    const int w = cells[3 * k + 2];
                    s_t[pos] = cells[3 * k + 1];
                    s_w[pos] = w;
                    s_c[pos] = sd > 0.0f ? gsnr[k] / (sd * sqrtf(static_cast<float>(w))) : 0.0f;
                }
            }
            cnt += __popc(bal);
        }
        __syncwarp();
        if (lane == 0) {
            if (cnt > kMaxCellsPerRow) atomicExch(err, 1);
            cnt = min(cnt, kMaxCellsPerRow);
            // row constants in cell order: sum_k -w_k c_k / N and -gsnr_k S_k / (N sd^2)
            int j = 0;
            for (int k = 0; k < n && j < cnt; ++k) {
                if (cells[3 * k] != d) continue;
                a += -static_cast<float>(s_w[j]) * s_c[j] / nf;
                if (sd > 0.0f) b += -gsnr[k] * snr[k] / (nf * sd * sd);
                ++j;
            }
            s_n = cnt;
            s_a = a;
            s_b = b;
        }
    }
    __syncthreads();
    const int cnt = s_n;
    const float a = s_a, b = s_b;
    const float* y = plane + static_cast<size_t>(d) * cols;
    float* g = gplane + static_cast<size_t>(d) * cols;
    for (int u = threadIdx.x; u < cols; u += blockDim.x) {
        float v = 0.0f;
        if (cnt > 0) {
            v = a + b * (__ldg(y + u) - m);
            for (int j = 0; j < cnt; ++j)
                if (u >= s_t[j] && u < s_t[j] + s_w[j]) v += s_c[j];
        }
        g[u] = v;
    }
}

inline int plane_pitch4(int ncols) { return (ncols + 31) / 32 * 32; }

size_t align256(size_t v) { return (v + 255) & ~static_cast<size_t>(255); }

// Rows of the adjoint's ping-pong planes: level l-1's gradient (l = niter..1)
// lives in buffer (l-1) & 1; the level-niter gradient is the caller's plane.
void adjoint_plane_rows(const FdmtPlanHost& h, size_t rows[2]) {
    rows[0] = rows[1] = 0;
    for (int l = 0; l < h.niter; ++l)
        rows[l & 1] = std::max(rows[l & 1], static_cast<size_t>(h.lv[l].total_rows()));
}

size_t adjoint_ws_bytes(const FdmtPlanHost& h) {
    size_t rows[2];
    adjoint_plane_rows(h, rows);
    const size_t P = plane_pitch4(h.ncols);
    return align256(rows[0] * P * sizeof(float)) + align256(rows[1] * P * sizeof(float));
}

bfs_status ensure_adjoint_tables(bfs_fdmt_plan* p) {
    if (p->d_adj_off) return BFS_OK;
    if (!p->adj.built) build_adjoint_tables(p->host, &p->adj);
    const AdjointTables& A = p->adj;
    BFS_CUDA(cudaMalloc(&p->d_adj_off, std::max<size_t>(1, A.off.size()) * sizeof(int)));
    BFS_CUDA(cudaMalloc(&p->d_adj_ent, std::max<size_t>(1, A.ent.size() / 2) * sizeof(int2)));
    if (!A.off.empty())
        BFS_CUDA(cudaMemcpy(p->d_adj_off, A.off.data(), A.off.size() * sizeof(int), cudaMemcpyHostToDevice));
    if (!A.ent.empty())
        BFS_CUDA(cudaMemcpy(p->d_adj_ent, A.ent.data(), A.ent.size() * sizeof(int), cudaMemcpyHostToDevice));
    return BFS_OK;
}

bfs_status adjoint_run(bfs_fdmt_plan* p, const float* d_gy, float* d_gx, float* buf0, float* buf1,
                       cudaStream_t s) {
    const FdmtPlanHost& h = p->host;
    const int T = h.ncols;
    const int P = plane_pitch4(T);
    float* bufs[2] = {buf0, buf1};
    const int span = kAdjThreads * kAdjVecs;
    const int gy_blocks = ((T + 3) / 4 + span - 1) / span;
    BFS_ARG(gy_blocks <= 65535, "ncols too large for this build");
    // Keith plans: the last merge level runs fused with the level-0 adjoint
    // when the level-1 gradient rows allow 16-byte reads
    const int r0c = h.rows_per_chan0;
    const float* src1 = (h.niter == 1) ? d_gy : bufs[1];
    const int pitch1 = (h.niter == 1) ? T : P;
    const bool fuse0 = h.kind == BFS_PLAN_KEITH && r0c >= 1 && r0c <= 5 && pitch1 % 4 == 0 &&
                       (reinterpret_cast<uintptr_t>(src1) & 15) == 0 &&
                       h.lv[0].total_rows() == h.nchan * r0c;
    for (int l = h.niter; l >= (fuse0 ? 2 : 1); --l) {
        const float* src = (l == h.niter) ? d_gy : bufs[l & 1];
        float* dst = bufs[(l - 1) & 1];
        const int in_pitch = (l == h.niter) ? T : P;
        const int rows_in = h.lv[l - 1].total_rows();
        const int* off = p->d_adj_off + p->adj.off_pos[l];
        const int2* ent = p->d_adj_ent + p->adj.ent_pos[l];
        dim3 grid(rows_in, gy_blocks);
        const bool vin = (in_pitch % 4 == 0) && (reinterpret_cast<uintptr_t>(src) & 15) == 0;
        if (vin)
            k_fdmt_adj_level<true><<<grid, kAdjThreads, 0, s>>>(src, dst, off, ent, T, in_pitch, P);
        else
            k_fdmt_adj_level<false><<<grid, kAdjThreads, 0, s>>>(src, dst, off, ent, T, in_pitch, P);
        BFS_LAUNCH_CHECK("k_fdmt_adj_level");
    }
    if (h.kind == BFS_PLAN_PRAVIR) {
        dim3 g2((T + kAdjInitThreads - 1) / kAdjInitThreads, h.nchan);
        BFS_ARG(g2.y <= 65535, "nchan too large for this build");
        k_fdmt_adj_init_grid<<<g2, kAdjInitThreads, 0, s>>>(bufs[0], d_gx, p->d_lvl0, h.nchan, T, P);
        BFS_LAUNCH_CHECK("k_fdmt_adj_init_grid");
        return BFS_OK;
    }
    const int vec_out = (T % 4 == 0) && (reinterpret_cast<uintptr_t>(d_gx) & 15) == 0;
    if (fuse0) {
        const int* off = p->d_adj_off + p->adj.off_pos[1];
        const int2* ent = p->d_adj_ent + p->adj.ent_pos[1];
        dim3 g0(((T + 3) / 4 + kAdjInitThreads - 2) / (kAdjInitThreads - 1), h.nchan);
        BFS_ARG(g0.y <= 65535, "nchan too large for this build");
        switch (r0c) {
            case 1: k_fdmt_adj_level0<1><<<g0, kAdjInitThreads, 0, s>>>(src1, d_gx, off, ent, T, pitch1, vec_out); break;
            case 2: k_fdmt_adj_level0<2><<<g0, kAdjInitThreads, 0, s>>>(src1, d_gx, off, ent, T, pitch1, vec_out); break;
            case 3: k_fdmt_adj_level0<3><<<g0, kAdjInitThreads, 0, s>>>(src1, d_gx, off, ent, T, pitch1, vec_out); break;
            case 4: k_fdmt_adj_level0<4><<<g0, kAdjInitThreads, 0, s>>>(src1, d_gx, off, ent, T, pitch1, vec_out); break;
            default: k_fdmt_adj_level0<5><<<g0, kAdjInitThreads, 0, s>>>(src1, d_gx, off, ent, T, pitch1, vec_out); break;
        }
        BFS_LAUNCH_CHECK("k_fdmt_adj_level0");
        return BFS_OK;
    }
    dim3 grid(((T + 3) / 4 + kAdjInitThreads - 1) / kAdjInitThreads, h.nchan);
    BFS_ARG(grid.y <= 65535, "nchan too large for this build");
    switch (h.rows_per_chan0) {
        case 1: k_fdmt_adj_init<1><<<grid, kAdjInitThreads, 0, s>>>(bufs[0], d_gx, T, P, 1, vec_out); break;
        case 2: k_fdmt_adj_init<2><<<grid, kAdjInitThreads, 0, s>>>(bufs[0], d_gx, T, P, 2, vec_out); break;
        case 3: k_fdmt_adj_init<3><<<grid, kAdjInitThreads, 0, s>>>(bufs[0], d_gx, T, P, 3, vec_out); break;
        case 4: k_fdmt_adj_init<4><<<grid, kAdjInitThreads, 0, s>>>(bufs[0], d_gx, T, P, 4, vec_out); break;
        case 5: k_fdmt_adj_init<5><<<grid, kAdjInitThreads, 0, s>>>(bufs[0], d_gx, T, P, 5, vec_out); break;
        default:
            k_fdmt_adj_init<0><<<grid, kAdjInitThreads, 0, s>>>(bufs[0], d_gx, T, P, h.rows_per_chan0, vec_out);
    }
    BFS_LAUNCH_CHECK("k_fdmt_adj_init");
    return BFS_OK;
}

}  // namespace
}  // namespace bfs

using namespace bfs;

extern "C" bfs_status bfs_fdmt_adjoint_workspace_size(const bfs_fdmt_plan* plan, size_t* bytes) {
    BFS_ARG(plan != nullptr && bytes != nullptr, "null argument");
    *bytes = adjoint_ws_bytes(plan->host);
    return BFS_OK;
}

extern "C" bfs_status bfs_fdmt_adjoint_ws(bfs_fdmt_plan* plan, const float* d_grad_out, float* d_grad_in,
                                          void* d_workspace, size_t workspace_bytes, void* stream) {
    BFS_ARG(plan != nullptr && d_grad_out != nullptr && d_grad_in != nullptr, "null argument");
    BFS_ARG(!plan->host_only, "plan was created with bfs_fdmt_plan_create_host");
    const size_t need = adjoint_ws_bytes(plan->host);
    BFS_ARG(d_workspace != nullptr && workspace_bytes >= need,
            "workspace of %zu bytes is smaller than the %zu needed", workspace_bytes, need);
    BFS_ARG((reinterpret_cast<uintptr_t>(d_workspace) & 255) == 0, "workspace must be 256-byte aligned");
    bfs_status st = ensure_adjoint_tables(plan);
    if (st != BFS_OK) return st;
    size_t rows[2];
    adjoint_plane_rows(plan->host, rows);
    char* w = static_cast<char*>(d_workspace);
    float* b0 = reinterpret_cast<float*>(w);
    float* b1 = reinterpret_cast<float*>(w + align256(rows[0] * plane_pitch4(plan->host.ncols) * sizeof(float)));
    return adjoint_run(plan, d_grad_out, d_grad_in, b0, b1, as_stream(stream));
}

extern "C" bfs_status bfs_fdmt_adjoint(bfs_fdmt_plan* plan, const float* d_grad_out, float* d_grad_in,
                                       void* stream) {
    BFS_ARG(plan != nullptr && d_grad_out != nullptr && d_grad_in != nullptr, "null argument");
    BFS_ARG(!plan->host_only, "plan was created with bfs_fdmt_plan_create_host");
    bfs_status st = ensure_adjoint_tables(plan);
    if (st != BFS_OK) return st;
    size_t rows[2];
    adjoint_plane_rows(plan->host, rows);
    const size_t P = plane_pitch4(plan->host.ncols);
    for (int b = 0; b < 2; ++b) {
        if (plan->d_adj_buf[b] || rows[b] == 0) continue;
        cudaError_t e = cudaMalloc(&plan->d_adj_buf[b], rows[b] * P * sizeof(float));
        if (e != cudaSuccess) {
            cudaGetLastError();
            plan->d_adj_buf[b] = nullptr;
            return fail(BFS_ERR_ALLOC, "cudaMalloc for an adjoint FDMT plane failed: %s", cudaGetErrorString(e));
        }
    }
    return adjoint_run(plan, d_grad_out, d_grad_in, static_cast<float*>(plan->d_adj_buf[0]),
                       static_cast<float*>(plan->d_adj_buf[1]), as_stream(stream));
}

extern "C" bfs_status bfs_boxcar_snr_cells(const float* d_plane, int rows, int cols, const float* d_stats,
                                           const int* d_cells, int n, float* d_snr, void* stream) {
    BFS_ARG(d_plane && d_stats && (n == 0 || (d_cells && d_snr)), "null argument");
    BFS_ARG(rows >= 1 && cols >= 1 && n >= 0, "bad shape");
    if (n == 0) return BFS_OK;
    k_snr_cells<<<(n + 127) / 128, 128, 0, as_stream(stream)>>>(d_plane, rows, cols, d_stats, d_cells, n, d_snr);
    BFS_LAUNCH_CHECK("k_snr_cells");
    return BFS_OK;
}

extern "C" bfs_status bfs_boxcar_snr_cells_adjoint(const float* d_plane, int rows, int cols,
                                                   const float* d_stats, const int* d_cells, int n,
                                                   const float* d_snr, const float* d_gsnr,
                                                   float* d_gplane, void* stream) {
    BFS_ARG(d_plane && d_stats && d_gplane && (n == 0 || (d_cells && d_snr && d_gsnr)), "null argument");
    BFS_ARG(rows >= 1 && cols >= 1 && n >= 0, "bad shape");
    cudaStream_t s = as_stream(stream);
    int* err = nullptr;
    bfs_status st = stream_alloc(reinterpret_cast<void**>(&err), sizeof(int), s);
    if (st != BFS_OK) return st;
    BFS_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
    k_snr_cells_adjoint<<<rows, 256, 0, s>>>(d_plane, rows, cols, d_stats, d_cells, n, d_snr, d_gsnr,
                                             d_gplane, err);
    BFS_LAUNCH_CHECK("k_snr_cells_adjoint");
    int h_err = 0;
    BFS_CUDA(cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, s));
    BFS_CUDA(cudaFreeAsync(err, s));
    BFS_CUDA(cudaStreamSynchronize(s));
    BFS_ARG(h_err == 0, "more than %d cells in one row", kMaxCellsPerRow);
    return BFS_OK;
}
