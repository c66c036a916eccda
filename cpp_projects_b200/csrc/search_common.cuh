// Device helpers shared by the search-stage kernels.
#pragma once

#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "bfs.h"

namespace bfs {

namespace cg = cooperative_groups;

constexpr int kStatCluster = 4;    // CTAs per row in the row-statistics kernels
constexpr int kStatThreads = 512;

// Per-row FP64 sum and sum of squares of x[row][0..cols), reduced across the
// kStatCluster CTAs of a thread-block cluster through distributed shared
// memory (deterministic order, no global scratch).  Returns the totals on
// cluster rank 0, thread 0; other threads get zeros.
__device__ inline void cluster_row_moments(const float* __restrict__ row, int cols, double& s_out,
                                           double& q_out) {
    __shared__ double sh_s[kStatThreads / 32], sh_q[kStatThreads / 32];
    __shared__ double part[2];
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = static_cast<int>(cluster.block_rank());
    const int per = (cols + kStatCluster - 1) / kStatCluster;
    const int beg = rank * per;
    const int end = min(cols, beg + per);
    double s = 0.0, q = 0.0;
    for (int t = beg + threadIdx.x; t < end; t += kStatThreads) {
        const double v = static_cast<double>(__ldg(row + t));
        s += v;
        q += v * v;
    }
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, o);
        q += __shfl_down_sync(0xffffffffu, q, o);
    }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) { sh_s[w] = s; sh_q[w] = q; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ts = 0.0, tq = 0.0;
        for (int i = 0; i < kStatThreads / 32; ++i) { ts += sh_s[i]; tq += sh_q[i]; }
        part[0] = ts; part[1] = tq;
    }
    cluster.sync();
    s_out = 0.0; q_out = 0.0;
    if (rank == 0 && threadIdx.x == 0) {
        for (int r = 0; r < kStatCluster; ++r) {
            const double* p = cluster.map_shared_rank(part, r);
            s_out += p[0];
            q_out += p[1];
        }
    }
    cluster.sync();  // keep every CTA's shared memory alive until rank 0 has read it
}

}  // namespace bfs
