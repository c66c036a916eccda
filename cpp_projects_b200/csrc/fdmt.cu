// FDMT on sm_100a.
//
// Reference semantics (L/FDMT/FdmtCpu.cpp:197-367, L/FDMT/FdmtGpu.cu:273-448):
//   level 0  row r of channel c at sample t is the running mean
//            v_r = (v_{r-1} * r + x[c][t-r]) / (r+1), v_0 = x[c][t], and 0 for t < r;
//   level l  out[g][t] = in[a_g][t] + (t >= s_g ? in[b_g][t - s_g] : 0), or a
//            copy of in[a_g] for the carried-over sub-band of an odd count.
// The products, sums and quotients use explicitly round-to-nearest intrinsics
// (no FMA contraction), so the result is bit-identical to the reference's CPU
// class run on one thread.
//
// Layout in HBM: every plane is row-major [row][ncols] float32, rows of a
// level concatenated sub-band by sub-band in frequency order (the reference's
// layout).  The plan owns two ping-pong planes sized for the largest even and
// odd level that reaches HBM, with rows padded to a 128-byte pitch so every
// merge level moves float4s whatever ncols is; the last level is written
// straight into the caller's output (pitch ncols).
//
// Reduced precision (opt-in, BFS_PREC_F16 / BFS_PREC_BF16): the planes that
// reach HBM between levels are stored as 16-bit values with a 128-byte row
// pitch; every sum is still formed in FP32 and the last level writes FP32.
// Row g of a stored plane holds v_g * 2^-e_g, e_g = ceil(log2(channels summed
// into row g)): a power-of-two per-row scale (exact, so it adds no rounding)
// that keeps the stored value within the input's own range (the row's channel
// mean), so FP16 cannot overflow where FP32 input fits FP16.  Levels inside
// the fused head stay FP32 in shared memory; only its output plane is stored.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>

#include "divide.cuh"
#include "internal.h"
#include "fdmt_plan.h"

namespace bfs {
namespace {

constexpr int kInitThreads = 256;
constexpr int kInitCols = 4;        // columns per thread (strided by the block)
constexpr int kLevelThreads = 256;

// 16-bit storage helpers.  The scale 2^e is built from its exponent bits
// (|e| < 127), so multiplying by it is exact.
__device__ __forceinline__ float to_f32(__half v) { return __half2float(v); }
__device__ __forceinline__ float to_f32(__nv_bfloat16 v) { return __bfloat162float(v); }
template <typename D> __device__ __forceinline__ D from_f32(float v);
template <> __device__ __forceinline__ float from_f32<float>(float v) { return v; }
template <> __device__ __forceinline__ __half from_f32<__half>(float v) { return __float2half_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 from_f32<__nv_bfloat16>(float v) {
    return __float2bfloat16_rn(v);
}
__device__ __forceinline__ unsigned bits16(__half v) { return __half_as_ushort(v); }
__device__ __forceinline__ unsigned bits16(__nv_bfloat16 v) { return __bfloat16_as_ushort(v); }
__device__ __forceinline__ float exp2_int(int e) { return __int_as_float((127 + e) << 23); }
// exponents packed in a table row's w: input a | input b << 8 | output << 16 (signed bytes)
__device__ __forceinline__ int exp_field(int w, int k) {
    return static_cast<int>(static_cast<signed char>((w >> (8 * k)) & 0xff));
}

// Level 0.  grid: (ceil(ncols / (256*4)), nchan).  D = float, or the 16-bit
// storage type (level-0 rows sum one channel: scale 2^0).
template <typename D>
__global__ void __launch_bounds__(kInitThreads)
k_fdmt_init(const float* __restrict__ x, D* __restrict__ out, int ncols, int out_pitch,
            int rows_per_chan, int ones) {
    const int c = blockIdx.y;
    const float* xr = x + static_cast<size_t>(c) * ncols;
    D* o = out + static_cast<size_t>(c) * rows_per_chan * out_pitch;
    const int base = blockIdx.x * (kInitThreads * kInitCols) + threadIdx.x;
#pragma unroll
    for (int k = 0; k < kInitCols; ++k) {
        const int t = base + k * kInitThreads;
        if (t >= ncols) break;
        float v = ones ? 1.0f : __ldg(xr + t);
        o[t] = from_f32<D>(v);
        for (int r = 1; r < rows_per_chan; ++r) {
            float w = 0.0f;
            if (t >= r) {
                const float xv = ones ? 1.0f : __ldg(xr + t - r);
                v = __fdiv_rn(__fadd_rn(__fmul_rn(v, static_cast<float>(r)), xv),
                              static_cast<float>(r + 1));
                w = v;
            }
            o[static_cast<size_t>(r) * out_pitch + t] = from_f32<D>(w);
        }
    }
}

// Level 0, 4 samples per thread (R0C = rows per channel, 1..5): thread q
// owns samples t = 4q .. 4q+3, reads them as one float4 (when the rows are
// 16-byte aligned) and the 4 before them from the lane below (warp shuffle;
// lane 0 loads its own), runs the 4 running means side by side and stores
// each row as one 16-byte (FP32) or 8-byte (16-bit) vector into the
// workspace plane (128-byte pitch; samples past ncols land in the pitch
// padding).  grid: (ceil(ceil(ncols / 4) / 256), nchan)
__device__ __forceinline__ float init_x(const float* __restrict__ xr, int tt, int ncols, int ones) {
    if (tt < 0 || tt >= ncols) return 0.0f;
    return ones ? 1.0f : __ldg(xr + tt);
}

template <typename D>
__device__ __forceinline__ void store4(D* __restrict__ p, const float (&v)[4]) {
    if constexpr (sizeof(D) == 4) {
        *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
    } else {
        const unsigned lo = bits16(from_f32<D>(v[0])) | (bits16(from_f32<D>(v[1])) << 16);
        const unsigned hi = bits16(from_f32<D>(v[2])) | (bits16(from_f32<D>(v[3])) << 16);
        *reinterpret_cast<uint2*>(p) = make_uint2(lo, hi);
    }
}

template <typename D, int R0C>
__global__ void __launch_bounds__(kInitThreads)
k_fdmt_init4(const float* __restrict__ x, D* __restrict__ out, int ncols, int out_pitch, int ones,
             int vec_x) {
    const int c = blockIdx.y;
    const float* xr = x + static_cast<size_t>(c) * ncols;
    D* o = out + static_cast<size_t>(c) * R0C * out_pitch;
    const int nv = (ncols + 3) >> 2;
    const int q = blockIdx.x * kInitThreads + threadIdx.x;
    const int t = 4 * q;
    const int lane = threadIdx.x & 31;
    float4 cur;
    if (vec_x && !ones && t + 3 < ncols)
        cur = __ldg(reinterpret_cast<const float4*>(xr) + q);
    else
        cur = make_float4(init_x(xr, t, ncols, ones), init_x(xr, t + 1, ncols, ones),
                          init_x(xr, t + 2, ncols, ones), init_x(xr, t + 3, ncols, ones));
    float4 prev;
    prev.x = __shfl_up_sync(0xffffffffu, cur.x, 1);
    prev.y = __shfl_up_sync(0xffffffffu, cur.y, 1);
    prev.z = __shfl_up_sync(0xffffffffu, cur.z, 1);
    prev.w = __shfl_up_sync(0xffffffffu, cur.w, 1);
    if (lane == 0)
        prev = make_float4(init_x(xr, t - 4, ncols, ones), init_x(xr, t - 3, ncols, ones),
                           init_x(xr, t - 2, ncols, ones), init_x(xr, t - 1, ncols, ones));
    if (q >= nv) return;
    const float xs[8] = {prev.x, prev.y, prev.z, prev.w, cur.x, cur.y, cur.z, cur.w};  // x[t-4 .. t+3]
    float v[4] = {cur.x, cur.y, cur.z, cur.w};
    store4<D>(o + t, v);
#pragma unroll
    for (int r = 1; r < R0C; ++r) {
        float w[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            w[j] = 0.0f;
            if (t + j >= r) {
                v[j] = div_small(__fadd_rn(__fmul_rn(v[j], static_cast<float>(r)), xs[4 + j - r]), r + 1);
                w[j] = v[j];
            }
        }
        store4<D>(o + static_cast<size_t>(r) * out_pitch + t, w);
    }
}

// Level 0 of a Pravir plan (L/FDMT_PRAVIR/fdmt_cpu.cpp:103-179): channel c
// has rows with delays dt_0 < dt_1 < ... (lvl0 = row cumsum over channels,
// then the delay of every row).  Row 0 at t >= dt_0 is the mean of
// x[t-dt_0 .. t]; row k at t >= dt_k is (row_{k-1} * (dt_{k-1} + 1) + the sum
// of x[t-dt_k .. t-dt_{k-1}-1]) / (dt_k + 1); earlier samples are 0.  Sums run
// in index order, one rounding per operation, as the reference.
// grid: (ceil(ncols / 256), nchan)
template <typename D>
__global__ void __launch_bounds__(kInitThreads)
k_fdmt_init_grid(const float* __restrict__ x, D* __restrict__ out, const int* __restrict__ lvl0,
                 int nchan, int ncols, int out_pitch, int ones) {
    const int c = blockIdx.y;
    const int t = blockIdx.x * kInitThreads + threadIdx.x;
    if (t >= ncols) return;
    const int r0 = __ldg(lvl0 + c), nr = __ldg(lvl0 + c + 1) - r0;
    const int* dts = lvl0 + nchan + 1 + r0;
    const float* xr = x + static_cast<size_t>(c) * ncols;
    D* o = out + static_cast<size_t>(r0) * out_pitch + t;
    float v = 0.0f;
    int dp = __ldg(dts);
    {
        float w = 0.0f;
        if (t >= dp) {
            float sum = 0.0f;
            for (int i = t - dp; i <= t; ++i) sum = __fadd_rn(sum, ones ? 1.0f : __ldg(xr + i));
            v = __fdiv_rn(sum, static_cast<float>(dp + 1));
            w = v;
        }
        o[0] = from_f32<D>(w);
    }
    for (int k = 1; k < nr; ++k) {
        const int dc = __ldg(dts + k);
        float w = 0.0f;
        if (t >= dc) {
            float sum = 0.0f;
            for (int i = t - dc; i < t - dp; ++i) sum = __fadd_rn(sum, ones ? 1.0f : __ldg(xr + i));
            v = __fdiv_rn(__fadd_rn(__fmul_rn(v, __fadd_rn(static_cast<float>(dp), 1.0f)), sum),
                          __fadd_rn(static_cast<float>(dc), 1.0f));
            w = v;
        }
        o[static_cast<size_t>(k) * out_pitch] = from_f32<D>(w);
        dp = dc;
    }
}

// Launches level 0 into a workspace plane (pitch P, 128-byte aligned rows).
template <typename D>
cudaError_t launch_init(const float* d_in, D* dst, const FdmtPlanHost& h, int P, int ones, cudaStream_t s,
                        const int* d_lvl0 = nullptr) {
    const int T = h.ncols;
    const int R = h.rows_per_chan0;
    if (h.kind == BFS_PLAN_PRAVIR) {
        dim3 grid((T + kInitThreads - 1) / kInitThreads, h.nchan);
        k_fdmt_init_grid<D><<<grid, kInitThreads, 0, s>>>(d_in, dst, d_lvl0, h.nchan, T, P, ones);
    } else if (R >= 1 && R <= 5) {
        dim3 grid(((T + 3) / 4 + kInitThreads - 1) / kInitThreads, h.nchan);
        const int vec_x = (T % 4 == 0) && d_in && (reinterpret_cast<uintptr_t>(d_in) & 15) == 0;
        switch (R) {
            case 1: k_fdmt_init4<D, 1><<<grid, kInitThreads, 0, s>>>(d_in, dst, T, P, ones, vec_x); break;
            case 2: k_fdmt_init4<D, 2><<<grid, kInitThreads, 0, s>>>(d_in, dst, T, P, ones, vec_x); break;
            case 3: k_fdmt_init4<D, 3><<<grid, kInitThreads, 0, s>>>(d_in, dst, T, P, ones, vec_x); break;
            case 4: k_fdmt_init4<D, 4><<<grid, kInitThreads, 0, s>>>(d_in, dst, T, P, ones, vec_x); break;
            default: k_fdmt_init4<D, 5><<<grid, kInitThreads, 0, s>>>(d_in, dst, T, P, ones, vec_x); break;
        }
    } else {
        dim3 grid((T + kInitThreads * kInitCols - 1) / (kInitThreads * kInitCols), h.nchan);
        k_fdmt_init<D><<<grid, kInitThreads, 0, s>>>(d_in, dst, T, P, R, ones);
    }
    return cudaGetLastError();
}

// FDMT of 0/1 rows (b_ones mode, or a plane whose row c is all w_c in {0,1}):
// output row d at sample t is exactly the number of channels c with w_c != 0
// and tau(d, c) <= t (the level-0 means of a 0/1 row are exactly 0 or 1 and
// every merge adds integers, so the level-by-level FDMT gives the same
// bits).  One CTA per output row: a shared histogram of tau over the row's
// channels (integer counts, exact in FP32), its inclusive prefix sum, then
// the row written once.  L = max tau + 1 histogram entries.
constexpr int kOnesThreads = 256;

__global__ void __launch_bounds__(kOnesThreads)
k_fdmt_ones(float* __restrict__ out, int out_pitch, const int* __restrict__ tau,
            const float* __restrict__ w, int w_stride, int nchan, int ncols, int L) {
    extern __shared__ float hist[];
    const int d = blockIdx.x;
    for (int i = threadIdx.x; i < L; i += blockDim.x) hist[i] = 0.0f;
    __syncthreads();
    const int* tr = tau + static_cast<size_t>(d) * nchan;
    for (int c = threadIdx.x; c < nchan; c += blockDim.x) {
        const bool on = w ? (__ldg(w + static_cast<size_t>(c) * w_stride) != 0.0f) : true;
        if (on) atomicAdd(&hist[__ldg(tr + c)], 1.0f);
    }
    __syncthreads();
    if (threadIdx.x < 32) {  // inclusive scan by one warp: a segment per lane
        const int lane = threadIdx.x;
        const int seg = (L + 31) / 32;
        const int b0 = min(L, lane * seg), b1 = min(L, b0 + seg);
        float sum = 0.0f;
        for (int i = b0; i < b1; ++i) sum += hist[i];
        float pre = sum;  // inclusive scan of the segment totals
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const float v = __shfl_up_sync(0xffffffffu, pre, o);
            if (lane >= o) pre += v;
        }
        float run = pre - sum;
        for (int i = b0; i < b1; ++i) {
            run += hist[i];
            hist[i] = run;
        }
    }
    __syncthreads();
    float* o = out + static_cast<size_t>(d) * out_pitch;
    const float last = hist[L - 1];
    for (int t = threadIdx.x; t < ncols; t += blockDim.x) o[t] = t < L ? hist[t] : last;
}

// One merge level.  The input plane is always a workspace plane (128-byte
// row pitch), so the tail row moves as float4; the shifted head row moves as
// 4 scalar loads (its alignment depends on the row's shift); the output is
// stored as float4 when its pitch and base allow (VOUT), else as scalars (the
// caller's plane with an odd ncols).  Each thread owns kLevelVecs column
// groups of 4 strided by the block.
// grid: (rows, ceil(ncols / (256*4*kLevelVecs)))
constexpr int kLevelVecs = 4;

template <bool VOUT>
__global__ void __launch_bounds__(kLevelThreads)
k_fdmt_level(const float* __restrict__ in, float* __restrict__ out, const int4* __restrict__ tab,
             int ncols, int in_pitch, int out_pitch) {
    const int g = blockIdx.x;
    const int4 e = __ldg(tab + g);
    const float4* ra = reinterpret_cast<const float4*>(in + static_cast<size_t>(e.x) * in_pitch);
    const float* rb = in + static_cast<size_t>(e.y < 0 ? e.x : e.y) * in_pitch;
    float* ro = out + static_cast<size_t>(g) * out_pitch;
    const int s = e.z;
    const bool has_b = e.y >= 0;
    const int nv = (ncols + 3) >> 2;
    const int base = blockIdx.y * (kLevelThreads * kLevelVecs) + threadIdx.x;
    float4 va[kLevelVecs];
    float vb[kLevelVecs][4];
#pragma unroll
    for (int k = 0; k < kLevelVecs; ++k) {
        const int q = base + k * kLevelThreads;
        va[k] = (q < nv) ? __ldg(ra + q) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int t = 4 * q + i;
            vb[k][i] = (has_b && t < ncols && t >= s) ? __ldg(rb + t - s) : 0.0f;
        }
    }
#pragma unroll
    for (int k = 0; k < kLevelVecs; ++k) {
        const int q = base + k * kLevelThreads;
        if (q >= nv) continue;
        const int t = 4 * q;
        float4 o = va[k];
        if (has_b) {
            if (t >= s) o.x = __fadd_rn(o.x, vb[k][0]);
            if (t + 1 >= s) o.y = __fadd_rn(o.y, vb[k][1]);
            if (t + 2 >= s) o.z = __fadd_rn(o.z, vb[k][2]);
            if (t + 3 >= s) o.w = __fadd_rn(o.w, vb[k][3]);
        }
        if (VOUT) {
            reinterpret_cast<float4*>(ro)[q] = o;
        } else {
            if (t < ncols) ro[t] = o.x;
            if (t + 1 < ncols) ro[t + 1] = o.y;
            if (t + 2 < ncols) ro[t + 2] = o.z;
            if (t + 3 < ncols) ro[t + 3] = o.w;
        }
    }
}

// One merge level over 16-bit planes (S = __half or __nv_bfloat16).  The
// input plane has a 128-byte pitch, so both rows move as aligned 8-element
// (16-byte) vectors: the tail row directly; the head row, shifted by s = 8*sv
// + r samples, as the aligned vector q - sv of each thread plus the one
// before it, taken from the neighbouring lane by a warp shuffle (lane 0
// loads its own), and the 8 wanted elements cut out of the pair with funnel
// shifts.  Both rows are widened to FP32 and rescaled by their rows' 2^e
// (exact); the sum is rounded once in FP32; the output is a 16-bit plane
// (D = S, 8-element vectors after scaling by 2^-e_out) or the caller's FP32
// plane (D = float, the last level).
// grid: (rows, ceil(ceil(ncols / 8) / (256 * kLevel16Vecs)))
constexpr int kLevel16Vecs = 2;

// words[0..7] = the 16 elements of vectors (q-sv-1, q-sv); out = elements
// P0..P0+7 (P0 = 8 - r, 1..7).
template <int P0>
__device__ __forceinline__ uint4 cut8(const uint32_t (&w)[8]) {
    uint32_t o[4];
    if constexpr ((P0 & 1) == 0) {
#pragma unroll
        for (int i = 0; i < 4; ++i) o[i] = w[P0 / 2 + i];
    } else {
#pragma unroll
        for (int i = 0; i < 4; ++i) o[i] = __funnelshift_r(w[P0 / 2 + i], w[P0 / 2 + i + 1], 16);
    }
    return make_uint4(o[0], o[1], o[2], o[3]);
}

__device__ __forceinline__ uint4 cut8(const uint32_t (&w)[8], int p0) {
    switch (p0) {
        case 1: return cut8<1>(w);
        case 2: return cut8<2>(w);
        case 3: return cut8<3>(w);
        case 4: return cut8<4>(w);
        case 5: return cut8<5>(w);
        case 6: return cut8<6>(w);
        default: return cut8<7>(w);
    }
}

template <typename S, typename D, bool VOUT>
__global__ void __launch_bounds__(kLevelThreads)
k_fdmt_level16(const S* __restrict__ in, D* __restrict__ out, const int4* __restrict__ tab,
               int ncols, int in_pitch, int out_pitch) {
    const int g = blockIdx.x;
    const int4 e = __ldg(tab + g);
    const float sa = exp2_int(exp_field(e.w, 0));
    const float sb = exp2_int(exp_field(e.w, 1));
    const float so = exp2_int(-exp_field(e.w, 2));
    const uint4* ra = reinterpret_cast<const uint4*>(in + static_cast<size_t>(e.x) * in_pitch);
    const uint4* rb = reinterpret_cast<const uint4*>(in + static_cast<size_t>(e.y < 0 ? e.x : e.y) * in_pitch);
    D* ro = out + static_cast<size_t>(g) * out_pitch;
    const int s = e.z;
    const int sv = s >> 3, r = s & 7;
    const bool has_b = e.y >= 0;
    const int nv = (ncols + 7) >> 3;
    const int lane = threadIdx.x & 31;
    const int base = blockIdx.y * (kLevelThreads * kLevel16Vecs) + threadIdx.x;
    const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
    uint4 va[kLevel16Vecs], vb[kLevel16Vecs];
#pragma unroll
    for (int k = 0; k < kLevel16Vecs; ++k) {
        const int q = base + k * kLevelThreads;
        va[k] = (q < nv) ? __ldg(ra + q) : zero;
        // head row: aligned vector q - sv (and q - sv - 1 when r > 0); the
        // shuffles run on every lane (warp-uniform: has_b and r are per row)
        const int qh = q - sv;
        uint4 hi = (has_b && qh >= 0 && qh < nv) ? __ldg(rb + qh) : zero;
        if (has_b && r != 0) {
            uint4 lo;
            lo.x = __shfl_up_sync(0xffffffffu, hi.x, 1);
            lo.y = __shfl_up_sync(0xffffffffu, hi.y, 1);
            lo.z = __shfl_up_sync(0xffffffffu, hi.z, 1);
            lo.w = __shfl_up_sync(0xffffffffu, hi.w, 1);
            if (lane == 0) lo = (qh - 1 >= 0 && qh - 1 < nv) ? __ldg(rb + qh - 1) : zero;
            const uint32_t w[8] = {lo.x, lo.y, lo.z, lo.w, hi.x, hi.y, hi.z, hi.w};
            hi = cut8(w, 8 - r);
        }
        vb[k] = hi;
    }
#pragma unroll
    for (int k = 0; k < kLevel16Vecs; ++k) {
        const int q = base + k * kLevelThreads;
        if (q >= nv) continue;
        const int t = 8 * q;
        const S* ha = reinterpret_cast<const S*>(&va[k]);
        const S* hb = reinterpret_cast<const S*>(&vb[k]);
        float o[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            o[i] = __fmul_rn(to_f32(ha[i]), sa);
            if (has_b && t + i >= s) o[i] = __fadd_rn(o[i], __fmul_rn(to_f32(hb[i]), sb));
        }
        if constexpr (sizeof(D) == 2) {
            uint4 pk;
            S* hp = reinterpret_cast<S*>(&pk);
#pragma unroll
            for (int i = 0; i < 8; ++i) hp[i] = from_f32<S>(__fmul_rn(o[i], so));
            reinterpret_cast<uint4*>(ro)[q] = pk;
        } else {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int t0 = t + 4 * h;
                if (VOUT && t0 + 4 <= ncols) {
                    reinterpret_cast<float4*>(ro + t0)[0] =
                        make_float4(o[4 * h], o[4 * h + 1], o[4 * h + 2], o[4 * h + 3]);
                } else {
#pragma unroll
                    for (int i = 0; i < 4; ++i)
                        if (t0 + i < ncols) ro[t0 + i] = o[4 * h + i];
                }
            }
        }
    }
}

// Fused levels 0..depth for one group of `group` adjacent channels and one
// tile of `tile` output samples.  blockDim.x = the tile plus the group's
// look-back (rounded to a warp): thread u owns sample t = tile0 - halo + u of
// every row.  Level 0 goes to shared buffer A, level 1 to B, level 2 to A, ...
// and the last level straight to the level-`depth` plane in HBM.  Only
// samples u >= halo are written; the plan's look-back guarantees that every
// value they depend on was computed from in-tile samples (u - shift >= 0), so
// the halo columns may hold partial values.  Samples t < 0 are the zeros the
// reference's planes hold there.  Buffer B first stages the group's input
// rows (it has at least `group` rows).  The group's row tables are staged in shared
// memory (after the two planes) and merge rows are processed four at a time
// with all loads issued before the stores.  R0C = level-0 rows per channel
// (0: runtime value rows_per_chan).
// grid: (ceil(ncols / tile), nchan / group)
// Level 0 of the group.  First every thread fetches its sample of each of
// the group's channel rows (all loads in flight at once, 8 per batch) into
// the staging rows of shared buffer B (free until level 1); then the running
// means read x[t - r] from there.  Local columns u - r < 0 (before the
// window) read 0: they lie in the halo, whose values never reach a written
// sample (the plan's look-back counts the level-0 window r).
template <int R0C>
__device__ __forceinline__ void head_level0(const float* __restrict__ x, float* __restrict__ bufa,
                                            float* __restrict__ stage, int c0, int group,
                                            int rows_per_chan, int ncols, int t, int u, int W,
                                            int ones) {
    constexpr int kBatch = 8;
    for (int cb = 0; cb < group; cb += kBatch) {
        float xv[kBatch];
#pragma unroll
        for (int k = 0; k < kBatch; ++k) {
            const int c = cb + k;
            xv[k] = 0.0f;
            if (c < group && t >= 0)
                xv[k] = ones ? 1.0f : (t < ncols ? __ldg(x + static_cast<size_t>(c0 + c) * ncols + t) : 0.0f);
        }
#pragma unroll
        for (int k = 0; k < kBatch; ++k)
            if (cb + k < group) stage[(cb + k) * W + u] = xv[k];
    }
    __syncthreads();
    const int r0c = R0C > 0 ? R0C : rows_per_chan;
#pragma unroll 2
    for (int c = 0; c < group; ++c) {
        const float* sx = stage + c * W + u;
        float* dst = bufa + c * r0c * W + u;
        float v = sx[0];
        dst[0] = v;
        if constexpr (R0C > 0) {
#pragma unroll
            for (int r = 1; r < R0C; ++r) {
                float w = 0.0f;
                if (t >= r) {
                    const float xr = u >= r ? sx[-r] : 0.0f;
                    // v * 1 is v: the first step needs no multiply
                    const float m = r == 1 ? v : __fmul_rn(v, static_cast<float>(r));
                    v = div_small(__fadd_rn(m, xr), r + 1);
                    w = v;
                }
                dst[r * W] = w;
            }
        } else {
#pragma unroll 1
            for (int r = 1; r < r0c; ++r) {
                float w = 0.0f;
                if (t >= r) {
                    const float xr = u >= r ? sx[-r] : 0.0f;
                    v = __fdiv_rn(__fadd_rn(__fmul_rn(v, static_cast<float>(r)), xr),
                                  static_cast<float>(r + 1));
                    w = v;
                }
                dst[r * W] = w;
            }
        }
    }
}

// One merge row of the head, from its staged entry {a, b, thr, d}: a = byte
// offset of the tail row in the source buffer, b = byte offset of the head
// row minus the shift (so b + 4u addresses sample u - shift), thr = the first
// local column that adds the head row (shift, raised by the samples t < 0 in
// the first tile), d = the destination offset.  `sb` = source buffer + u.
__device__ __forceinline__ float head_merge(const char* __restrict__ sb, int4 e, int u) {
    float a = *reinterpret_cast<const float*>(sb + e.x);
    if (u >= e.z) a = __fadd_rn(a, *reinterpret_cast<const float*>(sb + e.y));
    return a;
}

template <int R0C, typename D>
__global__ void __launch_bounds__(1024, 1)
k_fdmt_head(const float* __restrict__ x, D* __restrict__ out,
            const HeadGroup* __restrict__ groups, const int4* __restrict__ tab, int ncols,
            int out_pitch, int depth, int group, int rows_per_chan, int tile, int rows_a,
            int rows_b, int ones) {
    // a 16-bit output plane holds the level-`depth` rows (2^depth channels each) / 2^depth
    const float oscale = exp2_int(-depth);
    extern __shared__ float sm[];
    const int W = blockDim.x;
    const int u = threadIdx.x;
    const HeadGroup* hg = groups + blockIdx.y;
    const int halo = __ldg(&hg->halo);
    const int t0 = blockIdx.x * tile - halo;  // sample of local column 0
    const int t = t0 + u;
    float* bufa = sm;
    float* bufb = sm + rows_a * W;
    int4* stab = reinterpret_cast<int4*>(sm + (rows_a + rows_b) * W);

    // stage this group's tables (levels 1..depth are contiguous) as offsets:
    // t >= shift and u >= shift  <=>  u >= shift + max(0, -t0)
    const int tab0 = __ldg(&hg->tab_off[1]);
    const int last0 = __ldg(&hg->tab_off[depth]) - tab0;
    const int ntab = last0 + __ldg(&hg->rows[depth]);
    const int neg0 = max(0, -t0);
    for (int i = u; i < ntab; i += W) {
        const int4 e = __ldg(tab + tab0 + i);
        int l = 1;
        while (l < depth && i >= __ldg(&hg->tab_off[l + 1]) - tab0) ++l;
        const int j = i - (__ldg(&hg->tab_off[l]) - tab0);  // row within its level
        int4 f;
        f.x = e.x * W * 4;
        f.y = (e.y * W - e.z) * 4;
        f.z = e.z + neg0;
        f.w = l < depth ? j * W * 4 : j;
        stab[i] = f;
    }

    head_level0<R0C>(x, bufa, bufb, blockIdx.y * group, group, rows_per_chan, ncols, t, u, W, ones);
    __syncthreads();

    float* src = bufa;
    float* dst = bufb;
    const bool writer = (u >= halo) && (u < halo + tile) && (t < ncols);
    const int4* tb = stab;
    for (int l = 1; l <= depth; ++l) {
        const int rows = __ldg(&hg->rows[l]);
        const char* sb = reinterpret_cast<const char*>(src + u);
        if (l < depth) {
            char* db = reinterpret_cast<char*>(dst + u);
            int j = 0;
            for (; j + 4 <= rows; j += 4) {
                float v[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) v[k] = head_merge(sb, tb[j + k], u);
#pragma unroll
                for (int k = 0; k < 4; ++k) *reinterpret_cast<float*>(db + tb[j + k].w) = v[k];
            }
            for (; j < rows; ++j) {
                const int4 e = tb[j];
                *reinterpret_cast<float*>(db + e.w) = head_merge(sb, e, u);
            }
            __syncthreads();
            float* tmp = src; src = dst; dst = tmp;
        } else {
            D* o = out + static_cast<size_t>(__ldg(&hg->out_row0)) * out_pitch + t;
            auto put = [&](int row, float v) {
                if constexpr (sizeof(D) == 4) o[static_cast<size_t>(row) * out_pitch] = from_f32<D>(v);
                else o[static_cast<size_t>(row) * out_pitch] = from_f32<D>(__fmul_rn(v, oscale));
            };
            // shared-memory reads and global stores do not alias: the
            // compiler may hoist the loads of later rows above the stores
#pragma unroll 4
            for (int j = 0; j < rows; ++j) {
                const float v = head_merge(sb, tb[j], u);
                if (writer) put(j, v);
            }
        }
        tb += rows;
    }
}

template <typename D>
using HeadKernel = void (*)(const float*, D*, const HeadGroup*, const int4*, int, int, int, int,
                            int, int, int, int, int);

template <typename D>
HeadKernel<D> head_kernel_for(int rows_per_chan) {
    switch (rows_per_chan) {
        case 1: return k_fdmt_head<1, D>;
        case 2: return k_fdmt_head<2, D>;
        case 3: return k_fdmt_head<3, D>;
        case 4: return k_fdmt_head<4, D>;
        default: return k_fdmt_head<0, D>;
    }
}

// Launches the fused head with its shared-memory opt-in.
template <typename D>
cudaError_t launch_head(const HeadPlan& hp, const FdmtPlanHost& h, const float* d_in, D* dst,
                        int out_pitch, const HeadGroup* groups, const int* tab, int ones,
                        cudaStream_t s) {
    HeadKernel<D> kern = head_kernel_for<D>(h.rows_per_chan0);
    if (hp.smem_bytes > 48 * 1024) {
        // opt in once per (kernel, size) so later launches (also inside a
        // stream capture) make no attribute call
        static std::mutex mu;
        static std::map<std::pair<const void*, int>, size_t> done;
        int dev = 0;
        cudaGetDevice(&dev);
        std::lock_guard<std::mutex> lock(mu);
        size_t& have = done[{reinterpret_cast<const void*>(kern), dev}];
        if (have < hp.smem_bytes) {
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 static_cast<int>(hp.smem_bytes));
            if (e != cudaSuccess) return e;
            have = hp.smem_bytes;
        }
    }
    dim3 grid((h.ncols + hp.tile - 1) / hp.tile, h.nchan / hp.group);
    kern<<<grid, hp.width, hp.smem_bytes, s>>>(d_in, dst, groups, reinterpret_cast<const int4*>(tab),
                                               h.ncols, out_pitch, hp.depth, hp.group,
                                               h.rows_per_chan0,
                                               hp.tile, hp.rows_a, hp.rows_b, ones);
    return cudaGetLastError();
}

// Launches one merge level (vector stores when the output allows them).
cudaError_t launch_level(const float* src, float* dst, const int4* tab, int rows, int T,
                         int in_pitch, int out_pitch, cudaStream_t s) {
    const int span = kLevelThreads * kLevelVecs;
    dim3 grid(rows, ((T + 3) / 4 + span - 1) / span);
    if (grid.y > 65535) return cudaErrorInvalidConfiguration;
    const bool vout = (out_pitch % 4 == 0) && (reinterpret_cast<uintptr_t>(dst) & 15) == 0;
    if (vout)
        k_fdmt_level<true><<<grid, kLevelThreads, 0, s>>>(src, dst, tab, T, in_pitch, out_pitch);
    else
        k_fdmt_level<false><<<grid, kLevelThreads, 0, s>>>(src, dst, tab, T, in_pitch, out_pitch);
    return cudaGetLastError();
}

// Launches one merge level over 16-bit planes.
template <typename S, typename D>
cudaError_t launch_level16(const S* src, D* dst, const int4* tab, int rows, int T, int in_pitch,
                           int out_pitch, cudaStream_t s) {
    const int span = kLevelThreads * kLevel16Vecs;
    dim3 grid(rows, ((T + 7) / 8 + span - 1) / span);
    if (grid.y > 65535) return cudaErrorInvalidConfiguration;
    const bool vout = (out_pitch % 4 == 0) && (reinterpret_cast<uintptr_t>(dst) & 15) == 0;
    if (sizeof(D) == 2 || vout)
        k_fdmt_level16<S, D, true><<<grid, kLevelThreads, 0, s>>>(src, dst, tab, T, in_pitch, out_pitch);
    else
        k_fdmt_level16<S, D, false><<<grid, kLevelThreads, 0, s>>>(src, dst, tab, T, in_pitch, out_pitch);
    return cudaGetLastError();
}

constexpr size_t kSegSmemTwoPerSm = 113 * 1024;  // two CTAs of the segment kernel per SM

// Fused merge segment (levels l0+1..l1 over tiles of `rows` level-l1 rows x
// kSegTile samples; the layout and entries are described with SegPlan).
// Persistent: CTA b runs tiles b, b + gridDim.x, ... (tile w = row tile
// w % nrt at time tile w / nrt, so neighbouring CTAs share the rows at tile
// edges through L2).  A tile's entries and level-l0 rows are copied into
// shared memory with 16-byte asynchronous copies (each input row's window
// starts on a 16-byte boundary; pieces outside [0, ncols) are zero-filled
// and only reach columns no written sample depends on), issued for the NEXT
// tile before the current one is merged, so HBM loads overlap the merges.
// Each level merges the rows of the buffer below into the other buffer and
// level l1 goes straight to HBM:
//   out[u] = A[u + da] + (t >= shift ? B[u + db] : -)
// with one round-to-nearest add, so every written sample equals the
// level-by-level result bit for bit.  A warp merges whole rows, lanes on
// consecutive columns, so every shared access is one conflict-free
// wavefront whatever the offsets.
// Rows without a head row (odd sub-band counts) add the row of -0.0.
// grid: min(tiles, resident CTAs), block: THREADS
// 16-byte asynchronous copy to shared-window byte address s (src_bytes < 16:
// the rest is zero-filled; 0: nothing is read)
__device__ __forceinline__ void cp_async16(unsigned s, const void* gmem, int src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes)
                 : "memory");
}
// 16 bytes, the whole piece read
__device__ __forceinline__ void cp_async16_full(unsigned s, const void* gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
// 4-byte form (any 4-byte aligned addresses)
__device__ __forceinline__ void cp_async4(unsigned s, const void* gmem, int src_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// One work item: K consecutive 32-column chunks of one row of a level, from
// chunk c0, all shared loads issued before the stores.  rd / wr = the float
// offsets of the buffers of the level below and of this level (32-bit shared
// offsets, so every access is one LDS / STS with an immediate per chunk).
// FAST: every sample of the tile is at or past the row's head shift.
template <int K, bool FAST>
__device__ __forceinline__ void seg_chunks(float* __restrict__ sm, int rd, int wr, int4 q, int c0,
                                           int lane, int thr) {
    const int col = c0 * 32 + lane;
    const float* pa = sm + (rd + q.x + col);
    const float* pb = sm + (rd + q.y + col);
    float* pw = sm + (wr + q.w + col);
    float va[K], vb[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        va[k] = pa[32 * k];
        vb[k] = pb[32 * k];
    }
#pragma unroll
    for (int k = 0; k < K; ++k)
        pw[32 * k] = (FAST || col + 32 * k >= thr) ? __fadd_rn(va[k], vb[k]) : va[k];
}

// Two rows of a level (fast tiles: every sample at or past every head
// shift), all 4K shared loads of both rows issued before any store.
template <int K>
__device__ __forceinline__ void seg_rows2(float* __restrict__ sm, int rd, int wr, int4 q0, int4 q1, bool two,
                                          int lane) {
    const float* pa0 = sm + (rd + q0.x + lane);
    const float* pb0 = sm + (rd + q0.y + lane);
    float* pw0 = sm + (wr + q0.w + lane);
    const float* pa1 = sm + (rd + q1.x + lane);
    const float* pb1 = sm + (rd + q1.y + lane);
    float* pw1 = sm + (wr + q1.w + lane);
    float a0[K], b0[K], a1[K], b1[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        a0[k] = pa0[32 * k];
        b0[k] = pb0[32 * k];
    }
    if (two) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            a1[k] = pa1[32 * k];
            b1[k] = pb1[32 * k];
        }
    }
#pragma unroll
    for (int k = 0; k < K; ++k) pw0[32 * k] = __fadd_rn(a0[k], b0[k]);
    if (two) {
#pragma unroll
        for (int k = 0; k < K; ++k) pw1[32 * k] = __fadd_rn(a1[k], b1[k]);
    }
}

// Level-0 row r of a channel at K chunks: the reference's running mean
// v_0 = x[t], v_k = (v_{k-1} k + x[t-k]) / (k+1) (k = 1..r), one rounding per
// operation as in k_fdmt_init4, from the channel's staged samples (pa = the
// offset of x[t] for this lane's first column); 0 before sample r.
template <int R, int K, bool FAST>
__device__ __forceinline__ void seg_level0_chunks(float* __restrict__ sm, int pa, int pw, int col, int thr) {
    float v[K];
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = sm[pa + 32 * k];
#pragma unroll
    for (int r = 1; r <= R; ++r) {
        float x[K];
#pragma unroll
        for (int k = 0; k < K; ++k) x[k] = sm[pa + 32 * k - r];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const float m = r == 1 ? v[k] : __fmul_rn(v[k], static_cast<float>(r));
            v[k] = div_small(__fadd_rn(m, x[k]), r + 1);
        }
    }
#pragma unroll
    for (int k = 0; k < K; ++k) sm[pw + 32 * k] = (FAST || col + 32 * k >= thr) ? v[k] : 0.0f;
}

// One level-0 row of an input segment (entry {x offset, -, r + lead, dst | r << 20}).
template <int R0C, int NC, bool FAST>
__device__ __forceinline__ void seg_level0_row(float* __restrict__ sm, int rd, int wr, int4 q, int lane,
                                               int t0) {
    const int r = (q.w >> 20) & 15;
    const int pa = rd + q.x + lane, pw = wr + (q.w & 0xfffff) + lane;
    const int thr = q.z - t0;
    switch (r) {
        case 0: seg_level0_chunks<0, NC, FAST>(sm, pa, pw, lane, thr); break;
        case 1: if constexpr (R0C > 1) seg_level0_chunks<1, NC, FAST>(sm, pa, pw, lane, thr); break;
        case 2: if constexpr (R0C > 2) seg_level0_chunks<2, NC, FAST>(sm, pa, pw, lane, thr); break;
        case 3: if constexpr (R0C > 3) seg_level0_chunks<3, NC, FAST>(sm, pa, pw, lane, thr); break;
        default: if constexpr (R0C > 4) seg_level0_chunks<4, NC, FAST>(sm, pa, pw, lane, thr); break;
    }
}

struct SegArgs {
    const float* in;
    float* out;
    const SegTile* tiles;
    const int4* ent;
    int ncols, in_pitch, out_pitch, nlev, zx, zy, max_thr, y0, x1, ent_base, max_ent, nrt, total;
    int vec;   // input rows 16-byte aligned: 16-byte copies, else 4-byte copies
    int ones;  // the input is all ones (normalisation mode): no loads
};

template <int NC, int THREADS, int R0C>
__global__ void __launch_bounds__(THREADS, THREADS <= 256 ? 2 : 1) k_fdmt_seg(const SegArgs a) {
    static_assert(THREADS == 256 || THREADS == 512 || THREADS == 1024, "CTA size");
    constexpr int kOutCPH = kSegTile / 32;  // chunks of an output row
    constexpr int kWarps = THREADS / 32;
    constexpr int kPieces = NC * 8;  // 16-byte pieces per shared row
    extern __shared__ __align__(16) float sm[];
    const unsigned sbase = static_cast<unsigned>(__cvta_generic_to_shared(sm));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < NC * 32; i += THREADS) {
        sm[a.zx + i] = -0.0f;
        sm[a.y0 + a.zy + i] = -0.0f;
        sm[a.x1 + a.zx + i] = -0.0f;
    }

    // copies tile w's entries and input rows into buffer `buf` (0: X0, 1: X1);
    // each warp reads the entries of four of its rows at once, then issues
    // their pieces (a piece starts on a multiple of 4 samples, so it lies
    // wholly before sample 0 or wholly after it)
    // the tile's record {first entry, row counts}, two 16-byte loads
    auto tile_rec = [&](int rt, int4& lo, int4& hi) {
        const int4* t = reinterpret_cast<const int4*>(a.tiles + rt);
        lo = __ldg(t);
        hi = __ldg(t + 1);
    };
    const bool single = a.x1 == 0;  // one input buffer: load after merging
    constexpr int inw = kWarps;     // every warp issues its share of the copies
    const bool issuer = true;
    const int it = threadIdx.x;
    // entries of a tile into entry buffer eb (tile j uses buffer j % 3; single: 0)
    auto issue_ent = [&](int rt, int eb) {
        int4 lo, hi;
        tile_rec(rt, lo, hi);
        const int nent = lo.y + lo.z + lo.w + (a.nlev >= 3 ? hi.x : 0) + (a.nlev >= 4 ? hi.y : 0) +
                         (a.nlev >= 5 ? hi.z : 0) + (a.nlev >= 6 ? hi.w : 0);
        const int4* ge = a.ent + lo.x;
        const unsigned se = sbase + 4u * (a.ent_base + 4 * eb * a.max_ent);
        for (int i = it; i < nent; i += 32 * inw) cp_async16(se + 16u * i, ge + i, 16);
    };
    // input rows of a tile into X buffer `buf`, its row entries read from
    // entry buffer eb (already in shared memory)
    auto issue_rows = [&](int rt, int tt, int buf, int eb) {
        const int nin = __ldg(&a.tiles[rt].n[0]);
        const int t0 = tt * kSegTile;
        const int4* q4 = reinterpret_cast<const int4*>(sm + a.ent_base) + eb * a.max_ent;
        const unsigned x = sbase + 4u * (buf ? a.x1 : 0);
        if (a.ones) {  // the all-ones image: 1 inside [0, ncols), 0 outside
            for (int r = warp; r < nin; r += inw) {
                const int4 q = q4[r];
                const int ts = t0 - q.y;
                float* d = sm + (buf ? a.x1 : 0) + q.w;
                for (int c = lane; c < 32 * NC; c += 32) d[c] = (ts + c >= 0 && ts + c < a.ncols) ? 1.0f : 0.0f;
            }
        } else if (!a.vec) {  // unaligned rows: 4-byte copies
            for (int r = warp; r < nin; r += inw) {
                const int4 q = q4[r];
                const int ts = t0 - q.y;
                const float* src = a.in + static_cast<size_t>(q.x) * a.in_pitch;
                const unsigned dst = x + 4u * q.w;
                for (int c = lane; c < 32 * NC; c += 32) {
                    const int t = ts + c;
                    const bool in = t >= 0 && t < a.ncols;
                    cp_async4(dst + 4u * c, in ? src + t : src, in ? 4 : 0);
                }
            }
        } else {
            constexpr int kPerLane = (kPieces + 31) / 32;
            for (int r = warp; r < nin; r += inw) {
                const int4 q = q4[r];
                const int ts = t0 - q.y;  // the row's first sample
                const float* src = a.in + static_cast<size_t>(q.x) * a.in_pitch;
                const unsigned dst = x + 4u * q.w;
                if (ts >= 0 && ts + 4 * kPieces <= a.ncols) {  // the whole window lies in [0, ncols)
                    const float* s0 = src + ts + 4 * lane;
                    const unsigned d0 = dst + 16u * lane;
#pragma unroll
                    for (int k = 0; k < kPerLane; ++k)
                        if (k < kPerLane - 1 || lane + 32 * k < kPieces) cp_async16_full(d0 + 512u * k, s0 + 128 * k);
                } else {
                    for (int pc = lane; pc < kPieces; pc += 32) {
                        const int t = ts + 4 * pc;
                        const int bytes = t < 0 ? 0 : 4 * max(0, min(4, a.ncols - t));
                        cp_async16(dst + 16u * pc, bytes > 0 ? src + t : src, bytes);
                    }
                }
            }
        }
    };

    // tile w = (row tile w % nrt, time tile w / nrt), stepped by gridDim.x
    // without dividing per tile
    const int gq = static_cast<int>(gridDim.x) / a.nrt, gr = static_cast<int>(gridDim.x) % a.nrt;
    auto step = [&](int& rt, int& tt) {
        rt += gr;
        tt += gq;
        if (rt >= a.nrt) { rt -= a.nrt; ++tt; }
    };
    const int cw = warp, ncw = kWarps;  // merging warps
    auto level_sync = [&]() { __syncthreads(); };
    const int G = static_cast<int>(gridDim.x);
    int w = blockIdx.x;
    int rt = w % a.nrt, tt = w / a.nrt;  // this CTA's current tile
    // prologue: entries of the first two tiles, then the first tile's rows
    if (w < a.total && issuer) {
        issue_ent(rt, 0);
        if (!single && w + G < a.total) {
            int r1 = rt, t1 = tt;
            step(r1, t1);
            issue_ent(r1, 1);
        }
        cp_async_wait_all();
    }
    __syncthreads();
    if (w < a.total && issuer) issue_rows(rt, tt, 0, 0);
    for (int j = 0; w < a.total; ++j, w += G) {
        const int buf = single ? 0 : j & 1;
        const int eb = single ? 0 : j % 3;
        cp_async_wait_all();
        __syncthreads();  // this tile's rows (and the next tile's entries) are in; the previous tile is done
        int rn = rt, tn = tt;
        step(rn, tn);
        const bool more = w + G < a.total;
        if (!single && issuer) {
            if (w + 2 * G < a.total) {  // entries two tiles ahead
                int r2 = rn, t2 = tn;
                step(r2, t2);
                issue_ent(r2, (j + 2) % 3);
            }
            if (more) issue_rows(rn, tn, buf ^ 1, (j + 1) % 3);
        }
        int4 lo, hi;
        tile_rec(rt, lo, hi);
        const int nlv[kSegMaxLevels + 1] = {lo.y, lo.z, lo.w, hi.x, hi.y, hi.z, hi.w};
        const int t0 = tt * kSegTile;
        rt = rn;
        tt = tn;
        const int xo = buf ? a.x1 : 0;  // this tile's X buffer
        const int4* e = reinterpret_cast<const int4*>(sm + a.ent_base) + eb * a.max_ent + nlv[0];
        const bool fast = t0 >= a.max_thr;  // no sample of this tile precedes its head row's shift
#pragma unroll
        for (int lev = 1; lev < kSegMaxLevels; ++lev) {
            if (lev >= a.nlev) break;
            const int nl = nlv[lev];
            const int rd = (lev & 1) ? xo : a.y0;
            const int wr = (lev & 1) ? a.y0 : xo;
            if (R0C > 0 && lev == 1) {  // input segment: level 0 from the staged channels
                if (fast) {
                    for (int r = cw; r < nl; r += ncw) seg_level0_row<R0C, NC, true>(sm, rd, wr, e[r], lane, t0);
                } else {
                    for (int r = cw; r < nl; r += ncw) seg_level0_row<R0C, NC, false>(sm, rd, wr, e[r], lane, t0);
                }
            } else if (fast) {
                for (int r = cw; r < nl; r += 2 * ncw) {
                    const int r1 = r + ncw;
                    seg_rows2<NC>(sm, rd, wr, e[r], e[r1 < nl ? r1 : r], r1 < nl, lane);
                }
            } else {
                for (int r = cw; r < nl; r += ncw) {
                    const int4 q = e[r];
                    seg_chunks<NC, false>(sm, rd, wr, q, 0, lane, q.z - t0);
                }
            }
            e += nl;
            level_sync();
        }
        // level l1: kSegTile samples per row, straight to HBM (q.w is the plane row)
        int nl = nlv[1];
#pragma unroll
        for (int i = 2; i <= kSegMaxLevels; ++i)
            if (i == a.nlev) nl = nlv[i];
        const int rd = (a.nlev & 1) ? xo : a.y0;
        const bool clean = fast && t0 + kSegTile <= a.ncols;   // no shift test, no row end in this tile
        for (int r = cw; r < nl; r += ncw) {
            const int4 q = e[r];
            const int col = lane;
            const float* pa = sm + (rd + q.x + col);
            const float* pb = sm + (rd + q.y + col);
            float va[kOutCPH], vb[kOutCPH];
#pragma unroll
            for (int k = 0; k < kOutCPH; ++k) {
                va[k] = pa[32 * k];
                vb[k] = pb[32 * k];
            }
            float* dst = a.out + static_cast<size_t>(q.w) * a.out_pitch + t0 + col;
            if (clean) {
#pragma unroll
                for (int k = 0; k < kOutCPH; ++k) dst[32 * k] = __fadd_rn(va[k], vb[k]);
            } else {
                const int thr = q.z - t0;
                const int lim = a.ncols - t0 - col;  // samples of this row left from this lane's first
#pragma unroll
                for (int k = 0; k < kOutCPH; ++k)
                    if (32 * k < lim) dst[32 * k] = (fast || col + 32 * k >= thr) ? __fadd_rn(va[k], vb[k]) : va[k];
            }
        }
        if (single && more) {  // every warp is done with the buffers: load the next tile
            __syncthreads();
            issue_ent(rn, 0);
            cp_async_wait_all();
            __syncthreads();
            issue_rows(rn, tn, 0, 0);
        }
    }
}

template <int NC, int THREADS, int R0C>
cudaError_t launch_seg_nc(const SegPlan& sp, const SegArgs& args, cudaStream_t s) {
    auto kern = k_fdmt_seg<NC, THREADS, R0C>;
    // The shared-memory opt-in is one value per kernel and device: it only
    // ever grows (a smaller setting would refuse a later, larger launch).
    // Resident CTAs per SM are cached per (device, size).  Both happen on the
    // first launch of a size, which therefore comes before any stream capture.
    static std::mutex mu;
    static std::map<int, size_t> optin;
    static std::map<std::pair<int, size_t>, int> resident;
    int dev = 0;
    cudaGetDevice(&dev);
    int per_sm = 0, sms = 0;
    {
        std::lock_guard<std::mutex> lock(mu);
        size_t& have = optin[dev];
        if (have < sp.smem_bytes) {
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 static_cast<int>(sp.smem_bytes));
            if (e != cudaSuccess) return e;
            have = sp.smem_bytes;
        }
        auto it = resident.find({dev, sp.smem_bytes});
        if (it == resident.end()) {
            cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, THREADS, sp.smem_bytes);
            if (e != cudaSuccess) return e;
            if (per_sm < 1) return cudaErrorInvalidConfiguration;
            it = resident.emplace(std::make_pair(dev, sp.smem_bytes), per_sm).first;
        }
        per_sm = it->second;
    }
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    const int grid = std::min(args.total, sms * per_sm);
    kern<<<grid, THREADS, sp.smem_bytes, s>>>(args);
    return cudaGetLastError();
}

template <int NC, int R0C>
cudaError_t launch_seg_threads(const SegPlan& sp, const SegArgs& a, cudaStream_t s, int threads) {
    switch (threads) {
        case 256: return launch_seg_nc<NC, 256, R0C>(sp, a, s);
        case 512: return launch_seg_nc<NC, 512, R0C>(sp, a, s);
        case 1024: return launch_seg_nc<NC, 1024, R0C>(sp, a, s);
        default: return cudaErrorInvalidValue;
    }
}

template <int R0C>
cudaError_t launch_seg_nc_any(const SegPlan& sp, const SegArgs& a, cudaStream_t s, int threads) {
    switch (sp.nc) {
        case 9: return launch_seg_threads<9, R0C>(sp, a, s, threads);
        case 10: return launch_seg_threads<10, R0C>(sp, a, s, threads);
        case 12: return launch_seg_threads<12, R0C>(sp, a, s, threads);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_seg_r0c(const SegPlan& sp, const SegArgs& a, cudaStream_t s, int threads) {
    switch (sp.r0c) {
        case 0: return launch_seg_nc_any<0>(sp, a, s, threads);
        case 1: return launch_seg_nc_any<1>(sp, a, s, threads);
        case 2: return launch_seg_nc_any<2>(sp, a, s, threads);
        case 3: return launch_seg_nc_any<3>(sp, a, s, threads);
        case 4: return launch_seg_nc_any<4>(sp, a, s, threads);
        case 5: return launch_seg_nc_any<5>(sp, a, s, threads);
        default: return cudaErrorInvalidValue;
    }
}

// Launches one fused segment (sp.nc is one of the instantiated chunk counts;
// 256 threads when two CTAs fit an SM, else 512).
cudaError_t launch_seg(const SegPlan& sp, const float* src, float* dst, const SegTile* tiles,
                       const int4* ent, int T, int in_pitch, int out_pitch, cudaStream_t s, int ones = 0) {
    SegArgs a;
    a.in = src; a.out = dst; a.tiles = tiles; a.ent = ent;
    // 16-byte copies need 16-byte aligned rows (workspace planes always are;
    // a caller's filterbank when its base is and ncols % 4 == 0)
    a.vec = (in_pitch % 4 == 0 && (reinterpret_cast<uintptr_t>(src) & 15) == 0) ? 1 : 0;
    a.ones = ones;
    a.ncols = T; a.in_pitch = in_pitch; a.out_pitch = out_pitch;
    a.nlev = sp.l1 - sp.l0 + (sp.r0c > 0 ? 1 : 0); a.max_thr = sp.max_thr;
    a.zx = sp.rows_x * sp.pitch; a.zy = sp.rows_y * sp.pitch;
    a.y0 = sp.y0; a.x1 = sp.x1; a.ent_base = sp.ent_base; a.max_ent = sp.max_ent;
    a.nrt = static_cast<int>(sp.tiles.size());
    const long long total = static_cast<long long>(a.nrt) * ((T + kSegTile - 1) / kSegTile);
    if (total > (1LL << 30)) return cudaErrorInvalidConfiguration;
    a.total = static_cast<int>(total);
    int threads = sp.threads;
    if (threads == 0) threads = sp.smem_bytes <= kSegSmemTwoPerSm ? 256 : 512;
    return launch_seg_r0c(sp, a, s, threads);
}

// Row pitch (elements) of the workspace planes: ncols rounded up to 128 bytes.
inline int plane_pitch(int ncols, int elem_bytes = 4) {
    const int per = 128 / elem_bytes;
    return (ncols + per - 1) / per * per;
}
inline int elem_bytes_of(int precision) { return precision == BFS_PREC_F32 ? 4 : 2; }

constexpr int kHeadTile = 256;
constexpr size_t kHeadSmemTwoPerSm = 113 * 1024;  // two CTAs per SM
constexpr size_t kHeadSmemMax = 227 * 1024;

}  // namespace
}  // namespace bfs

using namespace bfs;

// Scale exponent of every row of every level: ceil(log2(channels summed into
// the row)); level-0 rows cover one channel, a merged row the channels of
// its two inputs, a carried-over row those of its one input.
static std::vector<std::vector<int>> row_exponents(const FdmtPlanHost& h) {
    std::vector<std::vector<int>> cnt(h.niter + 1), ex(h.niter + 1);
    cnt[0].assign(h.lv[0].total_rows(), 1);
    for (int l = 1; l <= h.niter; ++l) {
        const FdmtLevel& L = h.lv[l];
        cnt[l].resize(L.total_rows());
        for (int g = 0; g < L.total_rows(); ++g)
            cnt[l][g] = cnt[l - 1][L.a_row[g]] + (L.b_row[g] >= 0 ? cnt[l - 1][L.b_row[g]] : 0);
    }
    for (int l = 0; l <= h.niter; ++l) {
        ex[l].resize(cnt[l].size());
        for (size_t g = 0; g < cnt[l].size(); ++g) {
            int e = 0;
            while ((1 << e) < cnt[l][g]) ++e;
            ex[l][g] = e;
        }
    }
    return ex;
}

constexpr int kSegDefaultLevels = 3;

// The passes after the head (or level 0): levels k+1..niter cut into fused
// segments of about desc->seg_levels levels (FP32 plans), or one plain merge
// pass per level; then the ping-pong plane of every level that reaches HBM.
static bfs_status build_passes(const bfs_fdmt_desc* desc, bfs_fdmt_plan* p) {
    const FdmtPlanHost& h = p->host;
    const int k = p->head.depth;
    const int want = desc->seg_levels == 0 ? kSegDefaultLevels : desc->seg_levels;
    BFS_ARG(want >= 1 && want <= kSegMaxLevels, "seg_levels %d out of range (0..%d)", desc->seg_levels,
            kSegMaxLevels);
    BFS_ARG(desc->seg_rows >= 0, "seg_rows %d is negative", desc->seg_rows);
    const bool explicit_seg = desc->seg_levels >= 2 || desc->seg_rows > 0;
    BFS_ARG((desc->seg_flags & ~BFS_SEG_SINGLE_BUFFER) == 0, "unknown seg_flags 0x%x", desc->seg_flags);
    const bool single = (desc->seg_flags & BFS_SEG_SINGLE_BUFFER) != 0;
    BFS_ARG(desc->seg_threads == 0 || desc->seg_threads == 256 || desc->seg_threads == 512 ||
                desc->seg_threads == 1024,
            "seg_threads %d is not 0, 256, 512 or 1024", desc->seg_threads);
    BFS_ARG(!explicit_seg || p->precision == BFS_PREC_F32,
            "fused merge segments are implemented for FP32 plans");
    p->passes.clear();
    auto plain = [&](int l) {
        SegPlan sp;
        sp.l0 = l - 1;
        sp.l1 = l;
        p->passes.push_back(sp);
    };
    const int left = h.niter - k;
    if (want < 2 || p->precision != BFS_PREC_F32 || left < 2) {
        for (int l = k + 1; l <= h.niter; ++l) plain(l);
    } else {
        const int nseg = (left + want - 1) / want;
        int l0 = k;
        for (int i = 0; i < nseg; ++i) {
            const int l1 = l0 + left / nseg + (i < left % nseg ? 1 : 0);
            // no head: the first segment reads the channels and forms level 0
            // itself (no level-0 plane), where the plan's level 0 allows it
            if (i == 0 && k == 0 && h.kind == BFS_PLAN_KEITH && l1 >= 2) {
                bool ok = false;
                for (int G : {desc->seg_rows > 0 ? desc->seg_rows : 32, 16}) {
                    for (size_t limit : {kHeadSmemTwoPerSm, kHeadSmemMax}) {
                        SegPlan sp;
                        if (!ok && build_seg_plan(h, 0, l1, G, kSegTile, limit, &sp, true, single)) {
                            p->passes.push_back(std::move(sp));
                            ok = true;
                        }
                    }
                }
                if (ok) {
                    l0 = l1;
                    continue;
                }
            }
            if (l1 == l0 + 1) {
                plain(l1);
            } else {
                // rows per tile: the most that keep two CTAs per SM, else one
                std::vector<std::pair<int, size_t>> rows_try = {
                    {64, kHeadSmemTwoPerSm}, {32, kHeadSmemTwoPerSm}, {16, kHeadSmemTwoPerSm},
                    {32, kHeadSmemMax}, {16, kHeadSmemMax}, {8, kHeadSmemMax}};
                if (desc->seg_rows > 0) rows_try = {{desc->seg_rows, kHeadSmemMax}};
                bool ok = false;
                for (const auto& [G, limit] : rows_try) {
                    SegPlan sp;
                    if (build_seg_plan(h, l0, l1, G, kSegTile, limit, &sp, false, single)) {
                        p->passes.push_back(std::move(sp));
                        ok = true;
                        break;
                    }
                }
                BFS_ARG(ok || !explicit_seg, "seg_levels %d / seg_rows %d are not usable for this plan",
                        desc->seg_levels, desc->seg_rows);
                if (!ok)
                    for (int l = l0 + 1; l <= l1; ++l) plain(l);
            }
            l0 = l1;
        }
    }
    for (SegPlan& sp : p->passes) sp.threads = desc->seg_threads;
    // planes in HBM: level k (unless an input segment forms it on chip), then
    // every pass's output, alternating between the two buffers (the last
    // level goes to the caller's output)
    p->plane_buf.assign(h.niter + 1, -1);
    int b = 0;
    const bool in_seg = !p->passes.empty() && p->passes[0].r0c > 0;
    if (!in_seg) p->plane_buf[k] = b;
    else b = 1;
    for (const SegPlan& sp : p->passes) p->plane_buf[sp.l1] = (b ^= 1);
    p->buf_rows[0] = p->buf_rows[1] = 0;
    for (int l = k; l < h.niter; ++l)
        if (p->plane_buf[l] >= 0)
            p->buf_rows[p->plane_buf[l]] =
                std::max(p->buf_rows[p->plane_buf[l]], static_cast<size_t>(h.lv[l].total_rows()));
    return BFS_OK;
}

static bfs_status plan_host_part(const bfs_fdmt_desc* desc, std::unique_ptr<bfs_fdmt_plan>& p) {
    BFS_ARG(desc != nullptr, "null argument");
    BFS_ARG(desc->plan_kind == BFS_PLAN_KEITH || desc->plan_kind == BFS_PLAN_PRAVIR,
            "unsupported plan_kind %d", desc->plan_kind);
    BFS_ARG(desc->precision == BFS_PREC_F32 || desc->precision == BFS_PREC_F16 ||
                desc->precision == BFS_PREC_BF16,
            "unsupported precision %d", desc->precision);
    p.reset(new bfs_fdmt_plan);
    p->host_only = true;
    p->precision = desc->precision;
    if (desc->plan_kind == BFS_PLAN_PRAVIR) {
        BFS_ARG(desc->precision == BFS_PREC_F32, "16-bit planes are implemented for BFS_PLAN_KEITH only");
        BFS_ARG(desc->fuse_depth <= 0, "BFS_PLAN_PRAVIR has no fused head (fuse_depth %d)", desc->fuse_depth);
        bfs_status st = build_pravir_plan(desc->fmin, desc->fmax, desc->nchan, desc->ncols, desc->max_dt,
                                          desc->dt_step > 0 ? desc->dt_step : 1, desc->dt_min, &p->host);
        if (st != BFS_OK) return st;
        p->fuse_depth = 0;
        return build_passes(desc, p.get());
    }
    bfs_status st = build_fdmt_plan(desc->fmin, desc->fmax, desc->nchan, desc->ncols,
                                    desc->max_dt, &p->host);
    if (st != BFS_OK) return st;
    FdmtPlanHost& hm = p->host;
    hm.dt_out.resize(hm.max_dt);
    for (int r = 0; r < hm.max_dt; ++r) hm.dt_out[r] = r;
    const FdmtPlanHost& h = p->host;
    // fused head: explicit depth, or the deepest one that keeps two CTAs per SM
    const int tile = desc->head_tile > 0 ? desc->head_tile : kHeadTile;
    if (desc->fuse_depth != 0) {
        const int want = desc->fuse_depth < 0 ? kHeadMaxDepth : desc->fuse_depth;
        const size_t limit = desc->fuse_depth < 0 ? kHeadSmemTwoPerSm : kHeadSmemMax;
        for (int k = std::min(want, h.niter); k >= 1; --k) {
            HeadPlan hp;
            if (build_head_plan(h, k, tile, limit, &hp)) {
                p->head = std::move(hp);
                break;
            }
            if (desc->fuse_depth > 0) break;  // an explicit depth is not lowered silently
        }
        BFS_ARG(desc->fuse_depth <= 0 || p->head.depth == desc->fuse_depth,
                "fuse_depth %d is not usable for this plan", desc->fuse_depth);
    }
    p->fuse_depth = p->head.depth;
    return build_passes(desc, p.get());
}

static inline int bfs_fdmt_plan_depth_of(int d) { return d; }

// ---------------------------------------------------------------------------
// Autotuner: head depth and tile, or the first segment forming level 0, then
// segment length, rows per tile and input buffers per CTA, timed on the
// plan's own shape.
// ---------------------------------------------------------------------------
namespace {
struct TuneKey {
    int nchan, max_dt, cols_bucket, precision, kind, dt_min, dt_step;
    uint32_t fmin_bits, fmax_bits;
    bool operator<(const TuneKey& o) const {
        return std::tie(nchan, max_dt, cols_bucket, precision, kind, dt_min, dt_step, fmin_bits, fmax_bits) <
               std::tie(o.nchan, o.max_dt, o.cols_bucket, o.precision, o.kind, o.dt_min, o.dt_step,
                        o.fmin_bits, o.fmax_bits);
    }
};
struct TuneVal { int depth, tile, seg, rows, flags; float ms; };
std::mutex g_tune_mu;
std::map<TuneKey, TuneVal> g_tune;

TuneKey tune_key(const bfs_fdmt_desc& d) {
    TuneKey k{};
    k.nchan = d.nchan; k.max_dt = d.max_dt; k.precision = d.precision;
    k.kind = d.plan_kind; k.dt_min = d.dt_min; k.dt_step = d.dt_step;
    int b = 0;
    while ((1 << b) < d.ncols && b < 30) ++b;
    k.cols_bucket = b;
    std::memcpy(&k.fmin_bits, &d.fmin, 4);
    std::memcpy(&k.fmax_bits, &d.fmax, 4);
    return k;
}
}  // namespace

static bfs_status tune_fdmt(const bfs_fdmt_desc& base, TuneVal* best) {
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto it = g_tune.find(tune_key(base));
        if (it != g_tune.end()) { *best = it->second; return BFS_OK; }
    }
    struct Cand { int depth, tile, seg, rows, flags; };
    std::vector<Cand> cands;
    // one merge pass per level: head depth x head tile
    cands.push_back({0, 0, 1, 0, 0});
    for (int k : {2, 3, 4, 5})
        for (int tile : {256, 512}) cands.push_back({k, tile, 1, 0, 0});
    // fused merge segments of 2, 3 or 4 levels x 16-32 rows per tile (FP32):
    // after a head (16 or 32 rows), or forming level 0 in the first segment
    // with one or two input buffers per CTA (one buffer: half the input
    // staging, so two CTAs share an SM where two buffers allow one; 24 and 28
    // rows bring a single-buffered input segment under half an SM's shared
    // memory)
    if (base.precision == BFS_PREC_F32)
        for (int seg : {2, 3, 4})
            for (int rows : {16, 24, 28, 32}) {
                for (int flags : {0, static_cast<int>(BFS_SEG_SINGLE_BUFFER)}) cands.push_back({0, 0, seg, rows, flags});
                if (rows == 16 || rows == 32)
                    for (int k : {2, 3, 4}) cands.push_back({k, 256, seg, rows, 0});
            }
    const size_t in_n = static_cast<size_t>(base.nchan) * base.ncols;
    const size_t out_n = static_cast<size_t>(base.max_dt) * base.ncols;
    float *d_in = nullptr, *d_out = nullptr;
    void* ws = nullptr;
    size_t ws_bytes = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    TuneVal win{0, 0, 1, 0, 0, 1e30f};
    bfs_status st = BFS_OK;
    cudaStream_t s = nullptr;
    if (cudaMalloc(&d_in, in_n * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&d_out, out_n * sizeof(float)) != cudaSuccess ||
        cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        st = fail(BFS_ERR_ALLOC, "autotune: cannot allocate scratch for a %dx%d FDMT", base.nchan, base.ncols);
    }
    if (st == BFS_OK) cudaMemsetAsync(d_in, 0, in_n * sizeof(float), s);
    for (const Cand& c : cands) {
        if (st != BFS_OK) break;
        bfs_fdmt_desc d = base;
        d.fuse_depth = c.depth;
        d.head_tile = c.tile;
        d.seg_levels = c.seg;
        d.seg_rows = c.rows;
        d.seg_threads = 0;
        d.seg_flags = c.flags;
        d.flags = BFS_FDMT_EXTERNAL_WS;
        bfs_fdmt_plan* p = nullptr;
        if (bfs_fdmt_plan_create(&d, &p) != BFS_OK) continue;  // depth/tile not usable here
        size_t need = 0;
        bfs_fdmt_workspace_size(p, &need);
        if (need > ws_bytes) {
            if (ws) cudaFree(ws);
            ws = nullptr;
            if (cudaMalloc(&ws, need) != cudaSuccess) { bfs_fdmt_plan_destroy(p); ws_bytes = 0; continue; }
            ws_bytes = need;
        }
        float ms = 1e30f;
        // a segment length that fell back to plain levels duplicates seg = 1
        bool fused = false;
        for (const SegPlan& sp : p->passes) fused |= !sp.tiles.empty();
        if (c.seg > 1 && !fused) { bfs_fdmt_plan_destroy(p); continue; }
        bool ok = bfs_fdmt_execute_ws(p, d_in, d_out, 0, ws, ws_bytes, s) == BFS_OK;
        for (int rep = 0; rep < 2 && ok; ++rep) {
            cudaEventRecord(e0, s);
            ok = bfs_fdmt_execute_ws(p, d_in, d_out, 0, ws, ws_bytes, s) == BFS_OK;
            cudaEventRecord(e1, s);
            cudaEventSynchronize(e1);
            float t = 0.0f;
            cudaEventElapsedTime(&t, e0, e1);
            ms = std::min(ms, t);
        }
        bfs_fdmt_plan_destroy(p);
        if (ok && ms < win.ms) win = TuneVal{bfs_fdmt_plan_depth_of(c.depth), c.tile, c.seg, c.rows, c.flags, ms};
    }
    if (ws) cudaFree(ws);
    if (d_in) cudaFree(d_in);
    if (d_out) cudaFree(d_out);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaGetLastError();
    if (st != BFS_OK) return st;
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune[tune_key(base)] = win;
    *best = win;
    return BFS_OK;
}

extern "C" bfs_status bfs_fdmt_autotune_desc(const bfs_fdmt_desc* desc, bfs_fdmt_desc* tuned, float* ms) {
    BFS_ARG(desc != nullptr, "null argument");
    TuneVal v{};
    bfs_status st = tune_fdmt(*desc, &v);
    if (st != BFS_OK) return st;
    if (tuned) {
        *tuned = *desc;
        tuned->fuse_depth = v.depth;
        tuned->head_tile = v.tile;
        tuned->seg_levels = v.seg;
        tuned->seg_rows = v.rows;
        tuned->seg_threads = 0;
        tuned->seg_flags = v.flags;
    }
    if (ms) *ms = v.ms;
    return BFS_OK;
}

extern "C" bfs_status bfs_fdmt_autotune(const bfs_fdmt_desc* desc, int* depth, int* tile, float* ms) {
    bfs_fdmt_desc t{};
    bfs_status st = bfs_fdmt_autotune_desc(desc, &t, ms);
    if (st != BFS_OK) return st;
    if (depth) *depth = t.fuse_depth;
    if (tile) *tile = t.head_tile;
    return BFS_OK;
}

extern "C" bfs_status bfs_fdmt_plan_create_host(const bfs_fdmt_desc* desc, bfs_fdmt_plan** plan) {
    BFS_ARG(plan != nullptr, "null argument");
    *plan = nullptr;
    std::unique_ptr<bfs_fdmt_plan> p;
    bfs_status st = plan_host_part(desc, p);
    if (st != BFS_OK) return st;
    *plan = p.release();
    return BFS_OK;
}

extern "C" bfs_status bfs_fdmt_plan_create(const bfs_fdmt_desc* desc_in, bfs_fdmt_plan** plan) {
    BFS_ARG(plan != nullptr && desc_in != nullptr, "null argument");
    *plan = nullptr;
    bfs_fdmt_desc tuned = *desc_in;
    if (tuned.fuse_depth == BFS_FUSE_AUTOTUNE) {
        TuneVal v{};
        bfs_status ts = tune_fdmt(*desc_in, &v);
        if (ts != BFS_OK) return ts;
        tuned.fuse_depth = v.depth;
        tuned.head_tile = v.tile;
        tuned.seg_levels = v.seg;
        tuned.seg_rows = v.rows;
        tuned.seg_threads = 0;
        tuned.seg_flags = v.flags;
    }
    const bfs_fdmt_desc* desc = &tuned;
    std::unique_ptr<bfs_fdmt_plan> p;
    bfs_status st = plan_host_part(desc, p);
    if (st != BFS_OK) return st;
    p->host_only = false;
    BFS_CUDA(cudaGetDevice(&p->device));
    const FdmtPlanHost& h = p->host;
    if (p->head.depth > 0) {
        const HeadPlan& hp = p->head;
        BFS_CUDA(cudaMalloc(&p->d_head_groups, hp.groups.size() * sizeof(HeadGroup)));
        BFS_CUDA(cudaMemcpy(p->d_head_groups, hp.groups.data(),
                            hp.groups.size() * sizeof(HeadGroup), cudaMemcpyHostToDevice));
        BFS_CUDA(cudaMalloc(&p->d_head_tab, hp.tab.size() * sizeof(int)));
        BFS_CUDA(cudaMemcpy(p->d_head_tab, hp.tab.data(), hp.tab.size() * sizeof(int),
                            cudaMemcpyHostToDevice));
    }

    if (h.kind == BFS_PLAN_PRAVIR) {
        std::vector<int> l0(h.lv[0].cum.begin(), h.lv[0].cum.end());
        l0.insert(l0.end(), h.dt0.begin(), h.dt0.end());
        BFS_CUDA(cudaMalloc(&p->d_lvl0, l0.size() * sizeof(int)));
        BFS_CUDA(cudaMemcpy(p->d_lvl0, l0.data(), l0.size() * sizeof(int), cudaMemcpyHostToDevice));
    }
    // device row tables; with 16-bit planes w packs the per-row scale exponents
    const std::vector<std::vector<int>> ex = row_exponents(h);
    std::vector<int4> tab;
    p->tab_off.assign(h.niter + 1, 0);
    for (int l = 1; l <= h.niter; ++l) {
        p->tab_off[l] = tab.size();
        const FdmtLevel& L = h.lv[l];
        for (int g = 0; g < L.total_rows(); ++g) {
            int w = 0;
            if (p->precision != BFS_PREC_F32) {
                const int ea = ex[l - 1][L.a_row[g]];
                const int eb = L.b_row[g] >= 0 ? ex[l - 1][L.b_row[g]] : 0;
                const int eo = l == h.niter ? 0 : ex[l][g];
                w = (ea & 0xff) | ((eb & 0xff) << 8) | ((eo & 0xff) << 16);
            }
            tab.push_back(make_int4(L.a_row[g], L.b_row[g], L.shift[g], w));
        }
    }
    if (!tab.empty()) {
        BFS_CUDA(cudaMalloc(&p->d_tab, tab.size() * sizeof(int4)));
        BFS_CUDA(cudaMemcpy(p->d_tab, tab.data(), tab.size() * sizeof(int4),
                            cudaMemcpyHostToDevice));
    }
    // fused segments: every pass's tiles and entries, concatenated
    {
        std::vector<SegTile> tiles;
        std::vector<int> ent;
        p->seg_tile0.assign(p->passes.size(), 0);
        p->seg_ent0.assign(p->passes.size(), 0);
        for (size_t i = 0; i < p->passes.size(); ++i) {
            p->seg_tile0[i] = tiles.size();
            p->seg_ent0[i] = ent.size();
            tiles.insert(tiles.end(), p->passes[i].tiles.begin(), p->passes[i].tiles.end());
            ent.insert(ent.end(), p->passes[i].ent.begin(), p->passes[i].ent.end());
        }
        if (!tiles.empty()) {
            BFS_CUDA(cudaMalloc(&p->d_seg_tiles, tiles.size() * sizeof(SegTile)));
            BFS_CUDA(cudaMemcpy(p->d_seg_tiles, tiles.data(), tiles.size() * sizeof(SegTile),
                                cudaMemcpyHostToDevice));
            BFS_CUDA(cudaMalloc(&p->d_seg_ent, ent.size() * sizeof(int)));
            BFS_CUDA(cudaMemcpy(p->d_seg_ent, ent.data(), ent.size() * sizeof(int), cudaMemcpyHostToDevice));
        }
    }
    // ping-pong planes (sized by build_passes); levels inside the fused head
    // or a fused segment never reach HBM
    p->external_ws = (desc->flags & BFS_FDMT_EXTERNAL_WS) != 0;
    const int eb = elem_bytes_of(p->precision);
    for (int b = 0; b < 2 && !p->external_ws; ++b) {
        if (p->buf_rows[b] == 0) continue;
        const size_t bytes = p->buf_rows[b] * static_cast<size_t>(plane_pitch(h.ncols, eb)) * eb;
        cudaError_t e = cudaMalloc(&p->d_buf[b], bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            p->d_buf[b] = nullptr;
            return fail(BFS_ERR_ALLOC, "cudaMalloc(%zu) for an FDMT plane failed: %s", bytes,
                        cudaGetErrorString(e));
        }
        p->ws_bytes += bytes;
    }
    *plan = p.release();
    return BFS_OK;
}

extern "C" bfs_status bfs_fdmt_plan_destroy(bfs_fdmt_plan* plan) {
    delete plan;
    return BFS_OK;
}

extern "C" bfs_status bfs_fdmt_plan_head(const bfs_fdmt_plan* plan, int* params, int* groups,
                                         int group_cap, int* tab, int tab_cap) {
    BFS_ARG(plan != nullptr && params != nullptr, "null argument");
    const HeadPlan& hp = plan->head;
    params[0] = hp.depth; params[1] = hp.group; params[2] = hp.tile; params[3] = hp.width;
    params[4] = hp.rows_a; params[5] = hp.rows_b; params[6] = static_cast<int>(hp.smem_bytes);
    params[7] = static_cast<int>(hp.groups.size()); params[8] = static_cast<int>(hp.tab.size() / 4);
    const int gi = static_cast<int>(sizeof(HeadGroup) / sizeof(int));
    if (groups) {
        BFS_ARG(group_cap >= params[7] * gi, "groups needs %d ints", params[7] * gi);
        std::memcpy(groups, hp.groups.data(), hp.groups.size() * sizeof(HeadGroup));
    }
    if (tab) {
        BFS_ARG(tab_cap >= static_cast<int>(hp.tab.size()), "tab needs %zu ints", hp.tab.size());
        std::memcpy(tab, hp.tab.data(), hp.tab.size() * sizeof(int));
    }
    return BFS_OK;
}

extern "C" bfs_status bfs_fdmt_plan_passes(const bfs_fdmt_plan* plan, int* npasses, int* params, int cap) {
    BFS_ARG(plan != nullptr && npasses != nullptr, "null argument");
    const int n = static_cast<int>(plan->passes.size());
    *npasses = n;
    if (params) {
        BFS_ARG(cap >= 13 * n, "params needs %d ints", 13 * n);
        for (int i = 0; i < n; ++i) {
            const SegPlan& sp = plan->passes[i];
            const int v[13] = {sp.l0, sp.l1, sp.rows, sp.tile, sp.nc, sp.pitch, sp.rows_x, sp.rows_y,
                               sp.max_ent, sp.max_thr, static_cast<int>(sp.tiles.size()),
                               static_cast<int>(sp.ent.size() / 4), sp.r0c};
            std::memcpy(params + 13 * i, v, sizeof(v));
        }
    }
    return BFS_OK;
}

extern "C" bfs_status bfs_fdmt_plan_segment(const bfs_fdmt_plan* plan, int pass, int* tiles, int tiles_cap,
                                            int* ent, int ent_cap) {
    BFS_ARG(plan != nullptr, "null argument");
    BFS_ARG(pass >= 0 && pass < static_cast<int>(plan->passes.size()), "pass %d out of range", pass);
    const SegPlan& sp = plan->passes[pass];
    constexpr int ti = static_cast<int>(sizeof(SegTile) / sizeof(int));
    static_assert(ti == 8, "SegTile is 8 ints");
    if (tiles) {
        BFS_ARG(tiles_cap >= ti * static_cast<int>(sp.tiles.size()), "tiles needs %zu ints", ti * sp.tiles.size());
        std::memcpy(tiles, sp.tiles.data(), sp.tiles.size() * sizeof(SegTile));
    }
    if (ent) {
        BFS_ARG(ent_cap >= static_cast<int>(sp.ent.size()), "ent needs %zu ints", sp.ent.size());
        std::memcpy(ent, sp.ent.data(), sp.ent.size() * sizeof(int));
    }
    return BFS_OK;
}

// Bytes of the level-by-level algorithm: the input read, the level-0 plane
// written, each level's two input rows read and output row written per
// output row; intermediate planes of eb bytes per value, the output FP32.
static double fdmt_alg_bytes(const FdmtPlanHost& h, int precision) {
    const double eb = elem_bytes_of(precision);
    double bytes = 4.0 * h.nchan + eb * h.lv[0].total_rows();
    for (int l = 1; l <= h.niter; ++l)
        bytes += (l < h.niter ? 3.0 * eb : 2.0 * eb + 4.0) * h.lv[l].total_rows();
    return bytes * h.ncols;
}

extern "C" bfs_status bfs_fdmt_plan_info(const bfs_fdmt_plan* plan, bfs_fdmt_info* info) {
    BFS_ARG(plan != nullptr && info != nullptr, "null argument");
    const FdmtPlanHost& h = plan->host;
    info->niter = h.niter;
    info->rows_level0 = h.lv[0].total_rows();
    info->fuse_depth = plan->fuse_depth;
    int64_t tot = 0;
    for (const auto& L : h.lv) tot += L.total_rows();
    info->rows_total = tot;
    info->workspace_bytes = plan->ws_bytes;
    info->alg_bytes = fdmt_alg_bytes(h, plan->precision);
    info->out_rows = h.out_rows();
    info->hbm_passes = static_cast<int>(plan->passes.size());
    int seg = 1;
    for (const SegPlan& sp : plan->passes) seg = std::max(seg, sp.l1 - sp.l0);
    info->seg_levels = seg;
    // every plane that reaches HBM written once and read once, the input read,
    // the output written: the DRAM bytes this schedule cannot avoid
    const double eb = elem_bytes_of(plan->precision);
    double rows = 4.0 * h.nchan + 4.0 * h.out_rows();
    for (int l = 0; l < h.niter; ++l)
        if (!plan->plane_buf.empty() && plan->plane_buf[l] >= 0) rows += 2.0 * eb * h.lv[l].total_rows();
    info->sched_bytes = rows * h.ncols;
    return BFS_OK;
}

extern "C" bfs_status bfs_fdmt_plan_delays(const bfs_fdmt_plan* plan, int* out_dt, int out_cap,
                                           int* lvl0_cum, int* lvl0_dt, int lvl0_cap) {
    BFS_ARG(plan != nullptr, "null argument");
    const FdmtPlanHost& h = plan->host;
    if (out_dt) {
        BFS_ARG(out_cap >= h.out_rows(), "out_dt needs %d entries", h.out_rows());
        std::memcpy(out_dt, h.dt_out.data(), sizeof(int) * h.dt_out.size());
    }
    const int r0 = h.lv[0].total_rows();
    if (lvl0_cum) {
        BFS_ARG(lvl0_cap >= h.nchan + 1, "lvl0_cum needs %d entries", h.nchan + 1);
        std::memcpy(lvl0_cum, h.lv[0].cum.data(), sizeof(int) * (h.nchan + 1));
    }
    if (lvl0_dt) {
        BFS_ARG(lvl0_cap >= r0, "lvl0_dt needs %d entries", r0);
        for (int r = 0; r < r0; ++r)
            lvl0_dt[r] = h.kind == BFS_PLAN_PRAVIR ? h.dt0[r] : r % h.rows_per_chan0;
    }
    return BFS_OK;
}

extern "C" bfs_status bfs_fdmt_plan_rows(const bfs_fdmt_plan* plan, int* rows, int cap) {
    BFS_ARG(plan != nullptr && rows != nullptr, "null argument");
    BFS_ARG(cap >= plan->host.niter + 1, "need %d entries", plan->host.niter + 1);
    for (int l = 0; l <= plan->host.niter; ++l) rows[l] = plan->host.lv[l].total_rows();
    return BFS_OK;
}

extern "C" bfs_status bfs_fdmt_plan_tables(const bfs_fdmt_plan* plan, int level, int* a_row,
                                           int* b_row, int* shift, int cap) {
    BFS_ARG(plan != nullptr && a_row && b_row && shift, "null argument");
    BFS_ARG(level >= 1 && level <= plan->host.niter, "level %d out of range", level);
    const FdmtLevel& L = plan->host.lv[level];
    BFS_ARG(cap >= L.total_rows(), "need %d entries", L.total_rows());
    std::memcpy(a_row, L.a_row.data(), sizeof(int) * L.total_rows());
    std::memcpy(b_row, L.b_row.data(), sizeof(int) * L.total_rows());
    std::memcpy(shift, L.shift.data(), sizeof(int) * L.total_rows());
    return BFS_OK;
}

static size_t plane_bytes(const bfs_fdmt_plan* p, int b) {
    const int eb = elem_bytes_of(p->precision);
    const size_t raw = p->buf_rows[b] * static_cast<size_t>(plane_pitch(p->host.ncols, eb)) * eb;
    return (raw + 255) & ~static_cast<size_t>(255);
}

extern "C" bfs_status bfs_fdmt_workspace_size(const bfs_fdmt_plan* plan, size_t* bytes) {
    BFS_ARG(plan != nullptr && bytes != nullptr, "null argument");
    *bytes = plane_bytes(plan, 0) + plane_bytes(plan, 1);
    return BFS_OK;
}

constexpr int kOnesMaxHist = 12 * 1024;  // shared-memory histogram entries (48 KB)

// Uploads the plan's delay table for 0/1 rows on first use; false when the
// fast path does not apply (histogram too long).
static bfs_status ensure_ones(bfs_fdmt_plan* plan, bool* usable) {
    *usable = false;
    if (plan->ones_max_tau < 0) {
        std::vector<int> tau;
        int mx = 0;
        build_ones_delays(plan->host, &tau, &mx);
        plan->ones_max_tau = mx;
        if (mx + 1 <= kOnesMaxHist) {
            BFS_CUDA(cudaMalloc(&plan->d_ones_tau, tau.size() * sizeof(int)));
            BFS_CUDA(cudaMemcpy(plan->d_ones_tau, tau.data(), tau.size() * sizeof(int), cudaMemcpyHostToDevice));
        }
    }
    *usable = plan->d_ones_tau != nullptr;
    return BFS_OK;
}

static bfs_status launch_ones(bfs_fdmt_plan* plan, const float* d_w, int w_stride, float* d_out,
                              cudaStream_t s) {
    const FdmtPlanHost& h = plan->host;
    const int L = plan->ones_max_tau + 1;
    k_fdmt_ones<<<h.out_rows(), kOnesThreads, L * sizeof(float), s>>>(d_out, h.ncols, plan->d_ones_tau, d_w,
                                                                      w_stride, h.nchan, h.ncols, L);
    BFS_LAUNCH_CHECK("k_fdmt_ones");
    return BFS_OK;
}

// The same schedule over 16-bit planes (storage type S).
template <typename S>
static bfs_status fdmt_run16(bfs_fdmt_plan* plan, const float* d_in, float* d_out, int b_ones,
                             S* buf0, S* buf1, cudaStream_t s) {
    const FdmtPlanHost& h = plan->host;
    const int T = h.ncols;
    const int P = plane_pitch(T, 2);
    S* bufs[2] = {buf0, buf1};
    const int k = plan->head.depth;
    if (k > 0) {
        const HeadPlan& hp = plan->head;
        BFS_ARG(h.nchan / hp.group <= 65535, "nchan too large for this build");
        cudaError_t e = (k == h.niter)
            ? launch_head<float>(hp, h, d_in, d_out, T, plan->d_head_groups, plan->d_head_tab,
                                 b_ones ? 1 : 0, s)
            : launch_head<S>(hp, h, d_in, bufs[plan->plane_buf[k]], P, plan->d_head_groups,
                             plan->d_head_tab, b_ones ? 1 : 0, s);
        if (e != cudaSuccess) return fail(BFS_ERR_CUDA, "k_fdmt_head: %s", cudaGetErrorString(e));
    } else {
        BFS_ARG(h.nchan <= 65535, "nchan too large for this build");
        cudaError_t e = launch_init<S>(d_in, bufs[plan->plane_buf[0]], h, P, b_ones ? 1 : 0, s, plan->d_lvl0);
        if (e != cudaSuccess) return fail(BFS_ERR_CUDA, "k_fdmt_init: %s", cudaGetErrorString(e));
    }
    for (const SegPlan& sp : plan->passes) {  // 16-bit plans: one plain pass per level
        const int l = sp.l1;
        const S* src = bufs[plan->plane_buf[sp.l0]];
        const int4* tab = plan->d_tab + plan->tab_off[l];
        const int rows = h.lv[l].total_rows();
        cudaError_t e = (l == h.niter)
            ? launch_level16<S, float>(src, d_out, tab, rows, T, P, T, s)
            : launch_level16<S, S>(src, bufs[plan->plane_buf[l]], tab, rows, T, P, P, s);
        if (e != cudaSuccess) return fail(BFS_ERR_CUDA, "k_fdmt_level16: %s", cudaGetErrorString(e));
    }
    return BFS_OK;
}

static bfs_status fdmt_run(bfs_fdmt_plan* plan, const float* d_in, float* d_out, int b_ones,
                           void* buf0_, void* buf1_, cudaStream_t s) {
    if (plan->precision == BFS_PREC_F16)
        return fdmt_run16<__half>(plan, d_in, d_out, b_ones, static_cast<__half*>(buf0_),
                                  static_cast<__half*>(buf1_), s);
    if (plan->precision == BFS_PREC_BF16)
        return fdmt_run16<__nv_bfloat16>(plan, d_in, d_out, b_ones, static_cast<__nv_bfloat16*>(buf0_),
                                         static_cast<__nv_bfloat16*>(buf1_), s);
    if (b_ones) {
        bool usable = false;
        bfs_status st = ensure_ones(plan, &usable);
        if (st != BFS_OK) return st;
        if (usable) return launch_ones(plan, nullptr, 0, d_out, s);
    }
    float* buf0 = static_cast<float*>(buf0_);
    float* buf1 = static_cast<float*>(buf1_);
    const FdmtPlanHost& h = plan->host;
    const int T = h.ncols;
    const int P = plane_pitch(T);
    float* bufs[2] = {buf0, buf1};
    auto plane = [&](int l) { return l == h.niter ? d_out : bufs[plan->plane_buf[l]]; };
    auto pitch = [&](int l) { return l == h.niter ? T : P; };
    const int k = plan->head.depth;
    const bool in_seg = !plan->passes.empty() && plan->passes[0].r0c > 0;
    if (k > 0) {
        const HeadPlan& hp = plan->head;
        BFS_ARG(h.nchan / hp.group <= 65535, "nchan too large for this build");
        cudaError_t e = launch_head<float>(hp, h, d_in, plane(k), pitch(k), plan->d_head_groups,
                                           plan->d_head_tab, b_ones ? 1 : 0, s);
        if (e != cudaSuccess) return fail(BFS_ERR_CUDA, "k_fdmt_head: %s", cudaGetErrorString(e));
    } else if (in_seg) {
        // level 0 is formed by the first segment from the channels
    } else {
        BFS_ARG(h.nchan <= 65535, "nchan too large for this build");
        cudaError_t e = launch_init<float>(d_in, plane(0), h, P, b_ones ? 1 : 0, s, plan->d_lvl0);
        if (e != cudaSuccess) return fail(BFS_ERR_CUDA, "k_fdmt_init: %s", cudaGetErrorString(e));
    }
    for (size_t i = 0; i < plan->passes.size(); ++i) {
        const SegPlan& sp = plan->passes[i];
        const float* src = sp.r0c > 0 ? d_in : plane(sp.l0);
        cudaError_t e;
        if (sp.tiles.empty()) {
            e = launch_level(src, plane(sp.l1), plan->d_tab + plan->tab_off[sp.l1],
                             h.lv[sp.l1].total_rows(), T, P, pitch(sp.l1), s);
        } else if (sp.r0c > 0) {  // input segment: the caller's filterbank (pitch ncols)
            e = launch_seg(sp, d_in, plane(sp.l1), plan->d_seg_tiles + plan->seg_tile0[i],
                           reinterpret_cast<const int4*>(plan->d_seg_ent + plan->seg_ent0[i]), T, T,
                           pitch(sp.l1), s, b_ones ? 1 : 0);
        } else {
            e = launch_seg(sp, src, plane(sp.l1), plan->d_seg_tiles + plan->seg_tile0[i],
                           reinterpret_cast<const int4*>(plan->d_seg_ent + plan->seg_ent0[i]), T, P,
                           pitch(sp.l1), s);
        }
        if (e != cudaSuccess)
            return fail(BFS_ERR_CUDA, "%s (levels %d..%d): %s", sp.tiles.empty() ? "k_fdmt_level" : "k_fdmt_seg",
                        sp.l0 + 1, sp.l1, cudaGetErrorString(e));
    }
    return BFS_OK;
}

extern "C" bfs_status bfs_fdmt_execute(bfs_fdmt_plan* plan, const float* d_in, float* d_out,
                                       int b_ones, void* stream) {
    BFS_ARG(plan != nullptr && d_out != nullptr, "null argument");
    BFS_ARG(!plan->host_only, "plan was created with bfs_fdmt_plan_create_host");
    BFS_ARG(!plan->external_ws, "plan has no planes of its own: use bfs_fdmt_execute_ws");
    BFS_ARG(b_ones || d_in != nullptr, "d_in is null");
    return fdmt_run(plan, d_in, d_out, b_ones, plan->d_buf[0], plan->d_buf[1], as_stream(stream));
}

extern "C" bfs_status bfs_fdmt_execute_ws(bfs_fdmt_plan* plan, const float* d_in, float* d_out,
                                          int b_ones, void* d_workspace, size_t workspace_bytes,
                                          void* stream) {
    BFS_ARG(plan != nullptr && d_out != nullptr, "null argument");
    BFS_ARG(!plan->host_only, "plan was created with bfs_fdmt_plan_create_host");
    BFS_ARG(b_ones || d_in != nullptr, "d_in is null");
    const size_t need = plane_bytes(plan, 0) + plane_bytes(plan, 1);
    BFS_ARG(d_workspace != nullptr && workspace_bytes >= need,
            "workspace of %zu bytes is smaller than the %zu needed", workspace_bytes, need);
    BFS_ARG((reinterpret_cast<uintptr_t>(d_workspace) & 255) == 0, "workspace must be 256-byte aligned");
    char* w = static_cast<char*>(d_workspace);
    return fdmt_run(plan, d_in, d_out, b_ones, w, w + plane_bytes(plan, 0), as_stream(stream));
}

extern "C" bfs_status bfs_fdmt_execute_row_mask(bfs_fdmt_plan* plan, const float* d_mask, int mask_pitch,
                                                float* d_out, void* stream) {
    BFS_ARG(plan != nullptr && d_mask != nullptr && d_out != nullptr, "null argument");
    BFS_ARG(!plan->host_only, "plan was created with bfs_fdmt_plan_create_host");
    BFS_ARG(plan->precision == BFS_PREC_F32, "the row-mask FDMT is implemented for FP32 plans");
    bool usable = false;
    bfs_status st = ensure_ones(plan, &usable);
    if (st != BFS_OK) return st;
    BFS_ARG(usable, "the plan's delays exceed the row-mask histogram (%d)", kOnesMaxHist);
    return launch_ones(plan, d_mask, mask_pitch, d_out, as_stream(stream));
}

// ---------------------------------------------------------------------------
// Allocation-free FDMT.
//
// Some callers cannot allocate device memory when they need the transform: a
// real-time receiver that reserves all of its GPU memory at start-up and may
// not risk an allocation failure (or an allocator stall) mid-observation, a
// host framework that owns the device allocator and forbids side
// allocations, or a plain C caller linked against this library without its
// own CUDA allocation code.  bfs_fdmt_execute_noalloc serves them.  It takes
// a host-only plan (bfs_fdmt_plan_create_host: host memory only) and runs the
// same kernels as bfs_fdmt_execute, with every piece of scratch — the row
// tables and the two ping-pong planes — carved out of g_fdmt_static_scratch,
// a file-scope device array of kNoAllocScratchBytes (256 MiB) that every GPU
// which loads this library holds until the process exits.
//
// In host code the array's name is only a host-side stand-in, not a device
// address, so the device address is looked up with cudaGetSymbolAddress once
// per device (with that device current) on the first call made on it.  All calls
// share the one array and it keeps the previous call's contents: every byte a
// call reads is written by that call first (tables copied in, planes fully
// overwritten), so nothing needs clearing, but calls whose executions
// overlap on the GPU (other streams, other host threads) race on it.
// ---------------------------------------------------------------------------
#include <mutex>

namespace bfs {
namespace {

constexpr size_t kNoAllocScratchBytes = static_cast<size_t>(256) << 20;
constexpr int kNoAllocMaxDevices = 64;

__device__ __align__(256) unsigned char g_fdmt_static_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kNoAllocMaxDevices] = {};

bfs_status noalloc_scratch(void** out) {
    int dev = -1;
    BFS_CUDA(cudaGetDevice(&dev));
    BFS_ARG(dev >= 0 && dev < kNoAllocMaxDevices, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (g_noalloc_ptr[dev] == nullptr) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_fdmt_static_scratch);
        if (e != cudaSuccess || p == nullptr)
            return fail(BFS_ERR_CUDA, "cudaGetSymbolAddress(static FDMT scratch) on device %d: %s",
                        dev, cudaGetErrorString(e));
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return BFS_OK;
}

size_t align256(size_t v) { return (v + 255) & ~static_cast<size_t>(255); }

// Packs the three per-row int arrays staged in the scratch into int4 rows.
__global__ void k_pack_rows(const int* __restrict__ a, const int* __restrict__ b,
                            const int* __restrict__ s, int n, int4* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = make_int4(a[i], b[i], s[i], 0);
}

}  // namespace
}  // namespace bfs

extern "C" bfs_status bfs_fdmt_noalloc_scratch_bytes(const bfs_fdmt_plan* plan, size_t* need,
                                                     size_t* capacity) {
    BFS_ARG(plan != nullptr, "null argument");
    const FdmtPlanHost& h = plan->host;
    const int k = plan->head.depth;
    size_t rows = 0, prow[2] = {0, 0};
    for (int l = k + 1; l <= h.niter; ++l) rows += static_cast<size_t>(h.lv[l].total_rows());
    for (int l = k; l < h.niter; ++l)
        prow[l & 1] = std::max(prow[l & 1], static_cast<size_t>(h.lv[l].total_rows()));
    size_t total = align256(rows * sizeof(int4)) + align256(rows * 3 * sizeof(int));
    if (k > 0)
        total += align256(plan->head.groups.size() * sizeof(HeadGroup)) +
                 align256(plan->head.tab.size() * sizeof(int));
    const size_t P = static_cast<size_t>(plane_pitch(h.ncols));
    total += align256(prow[0] * P * sizeof(float)) + align256(prow[1] * P * sizeof(float));
    if (need) *need = total;
    if (capacity) *capacity = kNoAllocScratchBytes;
    return BFS_OK;
}

extern "C" bfs_status bfs_fdmt_execute_noalloc(const bfs_fdmt_plan* plan, const float* d_in,
                                               float* d_out, int b_ones, void* stream) {
    BFS_ARG(plan != nullptr && d_out != nullptr, "null argument");
    BFS_ARG(plan->precision == BFS_PREC_F32, "the allocation-free entry point runs FP32 plans only");
    BFS_ARG(plan->host.kind == BFS_PLAN_KEITH, "the allocation-free entry point runs BFS_PLAN_KEITH plans only");
    BFS_ARG(b_ones || d_in != nullptr, "d_in is null");
    size_t need = 0;
    bfs_status st = bfs_fdmt_noalloc_scratch_bytes(plan, &need, nullptr);
    if (st != BFS_OK) return st;
    BFS_ARG(need <= kNoAllocScratchBytes,
            "this FDMT needs %zu bytes of scratch; the allocation-free entry point has a fixed "
            "%zu-byte (256 MiB) static scratch: use bfs_fdmt_execute or bfs_fdmt_execute_ws",
            need, kNoAllocScratchBytes);
    void* base = nullptr;
    st = noalloc_scratch(&base);
    if (st != BFS_OK) return st;
    cudaStream_t s = as_stream(stream);
    const FdmtPlanHost& h = plan->host;
    const HeadPlan& hp = plan->head;
    const int k = hp.depth;
    const int T = h.ncols;

    // carve the scratch: packed tables | staged int tables | head groups | head table | planes
    char* p = static_cast<char*>(base);
    size_t rows = 0, prow[2] = {0, 0};
    for (int l = k + 1; l <= h.niter; ++l) rows += static_cast<size_t>(h.lv[l].total_rows());
    for (int l = k; l < h.niter; ++l)
        prow[l & 1] = std::max(prow[l & 1], static_cast<size_t>(h.lv[l].total_rows()));
    int4* tab = reinterpret_cast<int4*>(p);
    p += align256(rows * sizeof(int4));
    int* staged = reinterpret_cast<int*>(p);
    p += align256(rows * 3 * sizeof(int));
    HeadGroup* groups = nullptr;
    int* head_tab = nullptr;
    if (k > 0) {
        groups = reinterpret_cast<HeadGroup*>(p);
        p += align256(hp.groups.size() * sizeof(HeadGroup));
        head_tab = reinterpret_cast<int*>(p);
        p += align256(hp.tab.size() * sizeof(int));
    }
    float* bufs[2];
    bufs[0] = reinterpret_cast<float*>(p);
    const int P = plane_pitch(T);
    p += align256(prow[0] * static_cast<size_t>(P) * sizeof(float));
    bufs[1] = reinterpret_cast<float*>(p);

    // tables: host vectors -> staged ints -> packed int4 rows
    size_t off[64] = {};  // per level; niter <= 31 for any int channel count
    BFS_ARG(h.niter < 64, "too many levels");
    size_t pos = 0;
    for (int l = k + 1; l <= h.niter; ++l) {
        const FdmtLevel& L = h.lv[l];
        const size_t n = static_cast<size_t>(L.total_rows());
        off[l] = pos;
        BFS_CUDA(cudaMemcpyAsync(staged + pos, L.a_row.data(), n * sizeof(int), cudaMemcpyHostToDevice, s));
        BFS_CUDA(cudaMemcpyAsync(staged + rows + pos, L.b_row.data(), n * sizeof(int),
                                 cudaMemcpyHostToDevice, s));
        BFS_CUDA(cudaMemcpyAsync(staged + 2 * rows + pos, L.shift.data(), n * sizeof(int),
                                 cudaMemcpyHostToDevice, s));
        pos += n;
    }
    if (rows > 0) {
        const int n = static_cast<int>(rows);
        k_pack_rows<<<(n + 255) / 256, 256, 0, s>>>(staged, staged + rows, staged + 2 * rows, n, tab);
        BFS_LAUNCH_CHECK("k_pack_rows");
    }
    if (k > 0) {
        BFS_CUDA(cudaMemcpyAsync(groups, hp.groups.data(), hp.groups.size() * sizeof(HeadGroup),
                                 cudaMemcpyHostToDevice, s));
        BFS_CUDA(cudaMemcpyAsync(head_tab, hp.tab.data(), hp.tab.size() * sizeof(int),
                                 cudaMemcpyHostToDevice, s));
        BFS_ARG(h.nchan / hp.group <= 65535, "nchan too large for this build");
        float* dst = (k == h.niter) ? d_out : bufs[k & 1];
        cudaError_t e = launch_head<float>(hp, h, d_in, dst, (k == h.niter) ? T : P, groups,
                                           head_tab, b_ones ? 1 : 0, s);
        if (e != cudaSuccess) return fail(BFS_ERR_CUDA, "k_fdmt_head: %s", cudaGetErrorString(e));
    } else {
        BFS_ARG(h.nchan <= 65535, "nchan too large for this build");
        cudaError_t e = launch_init<float>(d_in, bufs[0], h, P, b_ones ? 1 : 0, s, plan->d_lvl0);
        if (e != cudaSuccess) return fail(BFS_ERR_CUDA, "k_fdmt_init: %s", cudaGetErrorString(e));
    }
    for (int l = k + 1; l <= h.niter; ++l) {
        const float* src = bufs[(l - 1) & 1];
        float* dst = (l == h.niter) ? d_out : bufs[l & 1];
        cudaError_t e = launch_level(src, dst, tab + off[l], h.lv[l].total_rows(), T, P,
                                     (l == h.niter) ? T : P, s);
        if (e != cudaSuccess) return fail(BFS_ERR_CUDA, "k_fdmt_level: %s", cudaGetErrorString(e));
    }
    return BFS_OK;
}
