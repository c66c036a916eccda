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

__global__ void k_clean_normalize(float* __restrict__ x, float* __restrict__ mask, int rows, int cols,
                                  const float* __restrict__ buff) {
    const int row = blockIdx.y;
    const float* g = buff + 2 * rows;
    const float mf = g[0], sf = g[1], dmf = g[2], dsf = g[3];
    const bool zap = static_cast<double>(fabsf(buff[rows + row] - dmf)) > 4.0 * static_cast<double>(dsf);
    const size_t base = static_cast<size_t>(row) * cols;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < cols; t += gridDim.x * blockDim.x) {
        if (zap) {
            x[base + t] = 0.0f;
            mask[base + t] = 0.0f;
        } else {
            x[base + t] = __fdiv_rn(__fsub_rn(x[base + t], mf), sf);
            mask[base + t] = 1.0f;
        }
    }
}

__global__ void k_fdmt_normalize(const float* __restrict__ f, const float* __restrict__ nrm, long long n,
                                 float* __restrict__ out) {
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const float den = __fsqrt_rn(__double2float_rn(static_cast<double>(nrm[i]) + 1.0e-8));
        out[i] = __fdiv_rn(f[i], den);
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
    dim3 grid(std::min((ncols + 255) / 256, 64), nrows);
    k_clean_normalize<<<grid, 256, 0, s>>>(d_inout, d_norm_input, nrows, ncols, d_buff);
    BFS_LAUNCH_CHECK("k_clean_normalize");
    return BFS_OK;
}

extern "C" bfs_status bfs_fdmt_normalize(const float* d_fdmt, const float* d_norm, int64_t n,
                                         float* d_out, void* stream) {
    BFS_ARG(d_fdmt && d_norm && d_out, "null argument");
    if (n <= 0) return BFS_OK;
    const long long blocks = std::min<long long>((n + 255) / 256, 148LL * 16);
    k_fdmt_normalize<<<static_cast<int>(blocks), 256, 0, as_stream(stream)>>>(d_fdmt, d_norm, n, d_out);
    BFS_LAUNCH_CHECK("k_fdmt_normalize");
    return BFS_OK;
}
