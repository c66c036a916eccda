// Statistical preprocessing of the FDMT input and the FDMT normalisation.
//
// Reference: statistical_preprocessing::calc_fdmt_inputs
// (L/CDMT/Statistical_preprocessing.cu:15-88) with its kernels
// calcRowMeanAndDisp (:278-329), kernel_OneSM_Mean_and_Std (:332-384),
// calculateMeanAndSTD_for_oneDimArray_kernel (:443-487) and
// normalize_clean_and_fill_NormInput (:510-539); fdmt_normalization
// (L/CDMT/Chunk_gpu.cu:842-852).
//
// The reference reduces in FP32 through single-block tree sums; here every
// reduction accumulates in FP64 (row moments in a 4-CTA cluster, the global
// moments in one block over the per-row values) and the results are rounded
// to float once, so the statistics sit at FP64 accuracy.  The scratch buffer
// keeps the reference's layout: [row mean][row variance][mean][std]
// [variance mean][variance std].
#include "internal.h"
#include "search_common.cuh"

namespace bfs {

bfs_status launch_row_stats(const float* d_in, int rows, int cols, float* d_stats, int mode,
                            cudaStream_t s);

namespace {

constexpr int kGlobalThreads = 1024;

__global__ void __launch_bounds__(kGlobalThreads)
k_global_stats(float* __restrict__ buff, int rows) {
    __shared__ double red[4][kGlobalThreads / 32];
    const float* rmean = buff;
    const float* rvar = buff + rows;
    double a = 0, b = 0, c = 0, d = 0;
    for (int r = threadIdx.x; r < rows; r += kGlobalThreads) {
        const double m = rmean[r], v = rvar[r];
        a += m;
        b += v + m * m;
        c += v;
        d += v * v;
    }
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
        c += __shfl_down_sync(0xffffffffu, c, o);
        d += __shfl_down_sync(0xffffffffu, d, o);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) { red[0][w] = a; red[1][w] = b; red[2][w] = c; red[3][w] = d; }
    __syncthreads();
    if (threadIdx.x == 0) {
        a = b = c = d = 0;
        for (int i = 0; i < kGlobalThreads / 32; ++i) { a += red[0][i]; b += red[1][i]; c += red[2][i]; d += red[3][i]; }
        const double mean = a / rows, var = b / rows - mean * mean;
        const double dmean = c / rows, dvar = d / rows - dmean * dmean;
        float* out = buff + 2 * rows;
        out[0] = static_cast<float>(mean);
        out[1] = static_cast<float>(sqrt(var > 0 ? var : 0.0));
        out[2] = static_cast<float>(dmean);
        out[3] = static_cast<float>(sqrt(dvar > 0 ? dvar : 0.0));
    }
}

__device__ __forceinline__ float clean_sample(float v, float mf, float sf) {
    return __fdiv_rn(__fsub_rn(v, mf), sf);
}

// VEC: cols % 4 == 0 and 16-byte aligned planes, so every row moves as float4s.
template <bool VEC>
__global__ void k_clean_normalize(float* __restrict__ x, float* __restrict__ mask, int rows, int cols,
                                  const float* __restrict__ buff) {
    const int row = blockIdx.y;
    const float* g = buff + 2 * rows;
    const float mf = g[0], sf = g[1], dmf = g[2], dsf = g[3];
    const bool zap = static_cast<double>(fabsf(buff[rows + row] - dmf)) > 4.0 * static_cast<double>(dsf);
    const size_t base = static_cast<size_t>(row) * cols;
    if constexpr (VEC) {
        float4* xr = reinterpret_cast<float4*>(x + base);
        float4* mr = reinterpret_cast<float4*>(mask + base);
        const int n4 = cols >> 2;
        const float4 z = make_float4(0.f, 0.f, 0.f, 0.f), one = make_float4(1.f, 1.f, 1.f, 1.f);
        for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n4; q += gridDim.x * blockDim.x) {
            if (zap) {
                xr[q] = z;
                mr[q] = z;
            } else {
                const float4 v = xr[q];
                xr[q] = make_float4(clean_sample(v.x, mf, sf), clean_sample(v.y, mf, sf),
                                    clean_sample(v.z, mf, sf), clean_sample(v.w, mf, sf));
                mr[q] = one;
            }
        }
    } else {
        for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < cols; t += gridDim.x * blockDim.x) {
            if (zap) {
                x[base + t] = 0.0f;
                mask[base + t] = 0.0f;
            } else {
                x[base + t] = clean_sample(x[base + t], mf, sf);
                mask[base + t] = 1.0f;
            }
        }
    }
}

__device__ __forceinline__ float fdmt_norm_sample(float f, float nrm) {
    const float den = __fsqrt_rn(__double2float_rn(static_cast<double>(nrm) + 1.0e-8));
    return __fdiv_rn(f, den);
}

// out = f / sqrtf((float)(nrm + 1e-8)); VEC: all three arrays 16-byte aligned,
// n4 = n / 4 float4 groups (the n % 4 tail is done by the scalar launch).
template <bool VEC>
__global__ void k_fdmt_normalize(const float* __restrict__ f, const float* __restrict__ nrm, long long n,
                                 float* __restrict__ out) {
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    const long long i0 = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if constexpr (VEC) {
        const float4* f4 = reinterpret_cast<const float4*>(f);
        const float4* n4p = reinterpret_cast<const float4*>(nrm);
        float4* o4 = reinterpret_cast<float4*>(out);
        const long long n4 = n >> 2;
        long long i = i0;
        for (; i + stride < n4; i += 2 * stride) {   // two groups in flight
            const float4 a = __ldg(f4 + i), b = __ldg(f4 + i + stride);
            const float4 ma = __ldg(n4p + i), mb = __ldg(n4p + i + stride);
            o4[i] = make_float4(fdmt_norm_sample(a.x, ma.x), fdmt_norm_sample(a.y, ma.y),
                                fdmt_norm_sample(a.z, ma.z), fdmt_norm_sample(a.w, ma.w));
            o4[i + stride] = make_float4(fdmt_norm_sample(b.x, mb.x), fdmt_norm_sample(b.y, mb.y),
                                         fdmt_norm_sample(b.z, mb.z), fdmt_norm_sample(b.w, mb.w));
        }
        if (i < n4) {
            const float4 a = __ldg(f4 + i), ma = __ldg(n4p + i);
            o4[i] = make_float4(fdmt_norm_sample(a.x, ma.x), fdmt_norm_sample(a.y, ma.y),
                                fdmt_norm_sample(a.z, ma.z), fdmt_norm_sample(a.w, ma.w));
        }
    } else {
        for (long long i = i0; i < n; i += stride) out[i] = fdmt_norm_sample(f[i], nrm[i]);
    }
}

}  // namespace
}  // namespace bfs

using namespace bfs;

extern "C" bfs_status bfs_preproc_calc_fdmt_inputs(float* d_inout, int nrows, int ncols,
                                                   float* d_buff, float* d_norm_input,
                                                   void* stream) {
    BFS_ARG(d_inout && d_buff && d_norm_input, "null argument");
    BFS_ARG(nrows >= 1 && ncols >= 1 && nrows <= 65535, "bad shape %dx%d", nrows, ncols);
    cudaStream_t s = as_stream(stream);
    bfs_status st = launch_row_stats(d_inout, nrows, ncols, d_buff, 1, s);
    if (st != BFS_OK) return st;
    k_global_stats<<<1, kGlobalThreads, 0, s>>>(d_buff, nrows);
    BFS_LAUNCH_CHECK("k_global_stats");
    const bool vec = (ncols % 4 == 0) && (reinterpret_cast<uintptr_t>(d_inout) & 15) == 0 &&
                     (reinterpret_cast<uintptr_t>(d_norm_input) & 15) == 0;
    if (vec) {
        dim3 grid(std::min((ncols / 4 + 255) / 256, 64), nrows);
        k_clean_normalize<true><<<grid, 256, 0, s>>>(d_inout, d_norm_input, nrows, ncols, d_buff);
    } else {
        dim3 grid(std::min((ncols + 255) / 256, 64), nrows);
        k_clean_normalize<false><<<grid, 256, 0, s>>>(d_inout, d_norm_input, nrows, ncols, d_buff);
    }
    BFS_LAUNCH_CHECK("k_clean_normalize");
    return BFS_OK;
}

extern "C" bfs_status bfs_fdmt_normalize(const float* d_fdmt, const float* d_norm, int64_t n,
                                         float* d_out, void* stream) {
    BFS_ARG(d_fdmt && d_norm && d_out, "null argument");
    if (n <= 0) return BFS_OK;
    cudaStream_t s = as_stream(stream);
    const bool vec = ((reinterpret_cast<uintptr_t>(d_fdmt) | reinterpret_cast<uintptr_t>(d_norm) |
                       reinterpret_cast<uintptr_t>(d_out)) & 15) == 0;
    if (vec && n >= 4) {
        const long long n4 = n / 4;
        const long long blocks = std::min<long long>((n4 + 255) / 256, 148LL * 8);
        k_fdmt_normalize<true><<<static_cast<int>(blocks), 256, 0, s>>>(d_fdmt, d_norm, n, d_out);
        BFS_LAUNCH_CHECK("k_fdmt_normalize");
        const long long done = n4 * 4;
        if (done < n)
            k_fdmt_normalize<false><<<1, 32, 0, s>>>(d_fdmt + done, d_norm + done, n - done, d_out + done);
    } else {
        const long long blocks = std::min<long long>((n + 255) / 256, 148LL * 16);
        k_fdmt_normalize<false><<<static_cast<int>(blocks), 256, 0, s>>>(d_fdmt, d_norm, n, d_out);
    }
    BFS_LAUNCH_CHECK("k_fdmt_normalize");
    return BFS_OK;
}
