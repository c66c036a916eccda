// Device helpers shared by the search-stage kernels.
#pragma once

#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "bfs.h"

namespace bfs {

namespace cg = cooperative_groups;

constexpr int kStatMaxCluster = 4;  // CTAs per row at most
constexpr int kStatThreads = 256;

// Per-row FP64 sum and sum of squares of x[row][0..cols), split over the
// CTAs of a thread-block cluster (its size set per launch) and reduced
// through distributed shared memory in rank order (deterministic, no global
// scratch).  CTA k of n reads samples [k per, (k + 1) per), per a multiple
// of 4.  The samples are taken in pieces of four from the first sample whose
// plane index (row_index cols + t) is a multiple of 4 — one 16-byte load
// each when the plane's base is 16-byte aligned (vec), four scalar loads
// otherwise — with the scalars before the first piece and after the last
// one thread each; every thread keeps four pieces in flight.  The assignment
// of samples to threads, and so the order of the additions, depends on the
// row's plane index only, not on where the plane lies in memory.  Returns the
// totals on cluster rank 0, thread 0; other threads get zeros.
__device__ inline void cluster_row_moments(const float* __restrict__ row, long long row_index, int cols,
                                           bool vec, double& s_out, double& q_out) {
    __shared__ double sh_s[kStatThreads / 32], sh_q[kStatThreads / 32];
    __shared__ double part[2];
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = static_cast<int>(cluster.block_rank());
    const int nb = static_cast<int>(cluster.num_blocks());
    const int per = ((cols + nb - 1) / nb + 3) & ~3;
    const int beg = min(cols, rank * per);
    const int end = min(cols, beg + per);
    // samples before the first piece: the plane index of `beg` up to a multiple of 4
    const int phase = static_cast<int>((row_index * cols + beg) & 3);
    const int lead = min(end - beg, (4 - phase) & 3);
    const int n4 = (end - beg - lead) >> 2;
    const float* p = row + beg + lead;
    auto piece = [&](int i) {
        if (vec) return __ldg(reinterpret_cast<const float4*>(p) + i);
        return make_float4(__ldg(p + 4 * i), __ldg(p + 4 * i + 1), __ldg(p + 4 * i + 2), __ldg(p + 4 * i + 3));
    };
    double s = 0.0, q = 0.0;
    auto add = [&](float4 v) {
        const double a = v.x, b = v.y, c = v.z, d = v.w;
        s += a; q += a * a;
        s += b; q += b * b;
        s += c; q += c * c;
        s += d; q += d * d;
    };
    int i = static_cast<int>(threadIdx.x);
    for (; i + 3 * kStatThreads < n4; i += 4 * kStatThreads) {
        const float4 v0 = piece(i), v1 = piece(i + kStatThreads);
        const float4 v2 = piece(i + 2 * kStatThreads), v3 = piece(i + 3 * kStatThreads);
        add(v0); add(v1); add(v2); add(v3);
    }
    for (; i < n4; i += kStatThreads) add(piece(i));
    // the lead scalars (threads 0..lead-1) and the tail ones (threads 4..6); lead < 4
    const int tail = end - beg - lead - 4 * n4;
    const int k = static_cast<int>(threadIdx.x);
    if (k < lead || (k >= 4 && k - 4 < tail)) {
        const double v = static_cast<double>(__ldg(k < lead ? row + beg + k : p + 4 * n4 + (k - 4)));
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
        for (int j = 0; j < kStatThreads / 32; ++j) { ts += sh_s[j]; tq += sh_q[j]; }
        part[0] = ts; part[1] = tq;
    }
    cluster.sync();
    s_out = 0.0; q_out = 0.0;
    if (rank == 0 && threadIdx.x == 0) {
        for (int r = 0; r < nb; ++r) {
            const double* pr = cluster.map_shared_rank(part, r);
            s_out += pr[0];
            q_out += pr[1];
        }
    }
    cluster.sync();  // keep every CTA's shared memory alive until rank 0 has read it
}

}  // namespace bfs
