// Candidate clustering and delegate selection on sm_100a.
//
// Reference: clusterization::complete_clusterization
// (L/Clusterization/Clusterization.cu:92-166) runs three grouping passes over
// the candidate fields mt, mdt and mwidth.  Each pass sorts the members of
// every current group by the field (sort_subarrays_cub_,
// L/Clusterization/Segmented_sort.cu:87-124) and starts a new group wherever
// two consecutive values differ by more than the pass's metric
// (calc_plan_and_values_for_regrouping_kernel / regrouping_kernel,
// Clusterization.cu:855-998).  A delegate is then picked per group
// (select_delegates_kernel, L/Clusterization/select_delegates.cu:63-125) and
// the delegates are sorted by mt (Clusterization.cu:147-149).
//
// Here one pass is: 64-bit key (group id << 32 | biased field value), a
// stable device radix sort of (key, candidate index) in index order — so ties
// resolve by candidate index, deterministically — a split-flag kernel, an
// inclusive scan of the flags (new group ids) and a scatter of the new ids.
// The reference's segmented sort is unstable; the group SETS it produces are
// the same (splits depend only on the sorted values), only the order inside
// a group differs, and the canonical order here is by candidate index.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <cfloat>
#include <climits>

#include "internal.h"

namespace bfs {
namespace {

constexpr int kDelegateLanes = 64;  // select_delegates_kernel's block size in the reference

__device__ __forceinline__ int field_of(const bfs_cand& c, int f) {
    return f == 0 ? c.mt : (f == 1 ? c.mdt : c.mwidth);
}

__device__ __forceinline__ unsigned biased(int v) { return static_cast<unsigned>(v) ^ 0x80000000u; }

__global__ void k_pass_keys(const bfs_cand* __restrict__ c, const unsigned* __restrict__ gid,
                            unsigned n, int field, unsigned long long* __restrict__ keys,
                            unsigned* __restrict__ vals) {
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned g = gid ? gid[i] : 0u;
    keys[i] = (static_cast<unsigned long long>(g) << 32) | biased(field_of(c[i], field));
    vals[i] = i;
}

__global__ void k_pass_flags(const bfs_cand* __restrict__ c, const unsigned long long* __restrict__ keys,
                             const unsigned* __restrict__ vals, unsigned n, int field,
                             long long metric, unsigned* __restrict__ flags) {
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    unsigned f = 1u;
    if (i > 0) {
        const unsigned g0 = static_cast<unsigned>(keys[i - 1] >> 32);
        const unsigned g1 = static_cast<unsigned>(keys[i] >> 32);
        if (g0 == g1) {
            const long long d = static_cast<long long>(field_of(c[vals[i]], field)) -
                                static_cast<long long>(field_of(c[vals[i - 1]], field));
            f = (d > metric) ? 1u : 0u;
        }
    }
    flags[i] = f;
}

__global__ void k_pass_scatter(const unsigned* __restrict__ vals, const unsigned* __restrict__ scan,
                               unsigned n, unsigned* __restrict__ gid) {
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) gid[vals[i]] = scan[i] - 1u;
}

__global__ void k_offsets(const unsigned* __restrict__ flags, const unsigned* __restrict__ scan,
                          unsigned n, int* __restrict__ offsets) {
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && flags[i]) offsets[scan[i] - 1u] = static_cast<int>(i);
    if (i == n - 1) offsets[scan[i]] = static_cast<int>(n);
}

// One block of 64 lanes per group: lane l scans members l, l+64, ... keeping
// the first strict maximum; the tree reduction keeps the lower lane on ties
// (the reference kernel's rule).
__global__ void __launch_bounds__(kDelegateLanes)
k_select_delegates(const bfs_cand* __restrict__ c, const int* __restrict__ perm, unsigned n,
                   const int* __restrict__ offsets, int* __restrict__ delegates) {
    __shared__ float sv[kDelegateLanes];
    __shared__ int si[kDelegateLanes];
    const int g = blockIdx.x;
    const int beg = offsets[g];
    const int len = offsets[g + 1] - beg;
    const int lane = threadIdx.x;
    float v = -FLT_MAX;
    int idx = lane;
    if (lane < len) {
        idx = -1;
        for (int i = lane; i < len; i += kDelegateLanes) {
            const int k = perm[beg + i];
            const float m = c[k].msnr;
            if (m > v) { v = m; idx = k; }
        }
    }
    sv[lane] = v;
    si[lane] = idx;
    __syncthreads();
    for (int s = kDelegateLanes / 2; s > 0; s >>= 1) {
        if (lane < s && sv[lane + s] > sv[lane]) { sv[lane] = sv[lane + s]; si[lane] = si[lane + s]; }
        __syncthreads();
    }
    if (lane == 0) delegates[g] = si[0];
}

__global__ void k_delegate_keys(const bfs_cand* __restrict__ c, const int* __restrict__ dl, unsigned ng,
                                unsigned long long* __restrict__ keys, unsigned* __restrict__ vals) {
    const unsigned g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ng) return;
    keys[g] = (static_cast<unsigned long long>(biased(c[dl[g]].mt)) << 32) | g;
    vals[g] = static_cast<unsigned>(dl[g]);
}

struct Scratch {
    cudaStream_t s;
    std::vector<void*> ptrs;
    bfs_status alloc(void** p, size_t bytes) {
        cudaError_t e = cudaMallocAsync(p, bytes ? bytes : 16, s);
        if (e != cudaSuccess) return fail(BFS_ERR_ALLOC, "cudaMallocAsync(%zu): %s", bytes,
                                          cudaGetErrorString(e));
        ptrs.push_back(*p);
        return BFS_OK;
    }
    ~Scratch() { for (void* p : ptrs) cudaFreeAsync(p, s); }
};

#define BFS_TRY(x) do { bfs_status st_ = (x); if (st_ != BFS_OK) return st_; } while (0)

}  // namespace
}  // namespace bfs

using namespace bfs;

extern "C" bfs_status bfs_select_delegates(const bfs_cand* d_cands, const int* d_perm, uint32_t n,
                                           const int* d_offsets, uint32_t ngroups,
                                           int* d_delegates, void* stream) {
    BFS_ARG(d_cands && d_perm && d_offsets && d_delegates, "null argument");
    if (ngroups == 0) return BFS_OK;
    BFS_ARG(n > 0, "groups without candidates");
    k_select_delegates<<<ngroups, kDelegateLanes, 0, as_stream(stream)>>>(d_cands, d_perm, n,
                                                                           d_offsets, d_delegates);
    BFS_LAUNCH_CHECK("k_select_delegates");
    return BFS_OK;
}

extern "C" bfs_status bfs_cluster(const bfs_cand* d_cands, uint32_t n, const int* metrics,
                                  int* d_perm, int* d_offsets, int* d_delegates,
                                  uint32_t* h_ngroups, void* stream) {
    BFS_ARG(metrics && h_ngroups, "null argument");
    *h_ngroups = 0;
    if (n == 0) return BFS_OK;
    BFS_ARG(d_cands && d_perm && d_offsets && d_delegates, "null argument");
    BFS_ARG(n < 0x7fffffffu, "too many candidates");
    cudaStream_t s = as_stream(stream);
    Scratch sc{s, {}};
    unsigned long long *k_in, *k_out;
    unsigned *v_in, *v_out, *gid, *flags, *scan;
    BFS_TRY(sc.alloc(reinterpret_cast<void**>(&k_in), sizeof(unsigned long long) * n));
    BFS_TRY(sc.alloc(reinterpret_cast<void**>(&k_out), sizeof(unsigned long long) * n));
    BFS_TRY(sc.alloc(reinterpret_cast<void**>(&v_in), sizeof(unsigned) * n));
    BFS_TRY(sc.alloc(reinterpret_cast<void**>(&v_out), sizeof(unsigned) * n));
    BFS_TRY(sc.alloc(reinterpret_cast<void**>(&gid), sizeof(unsigned) * n));
    BFS_TRY(sc.alloc(reinterpret_cast<void**>(&flags), sizeof(unsigned) * n));
    BFS_TRY(sc.alloc(reinterpret_cast<void**>(&scan), sizeof(unsigned) * n));
    size_t sort_bytes = 0, scan_bytes = 0;
    BFS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, k_in, k_out, v_in, v_out,
                                             static_cast<int>(n), 0, 64, s));
    BFS_CUDA(cub::DeviceScan::InclusiveSum(nullptr, scan_bytes, flags, scan, static_cast<int>(n), s));
    void* tmp;
    size_t tmp_bytes = std::max(sort_bytes, scan_bytes);
    BFS_TRY(sc.alloc(&tmp, tmp_bytes));
    const int th = 256;
    const int bl = static_cast<int>((n + th - 1) / th);
    for (int field = 0; field < 3; ++field) {
        k_pass_keys<<<bl, th, 0, s>>>(d_cands, field == 0 ? nullptr : gid, n, field, k_in, v_in);
        BFS_LAUNCH_CHECK("k_pass_keys");
        size_t b = tmp_bytes;
        BFS_CUDA(cub::DeviceRadixSort::SortPairs(tmp, b, k_in, k_out, v_in, v_out,
                                                 static_cast<int>(n), 0, 64, s));
        k_pass_flags<<<bl, th, 0, s>>>(d_cands, k_out, v_out, n, field,
                                       static_cast<long long>(metrics[field]), flags);
        BFS_LAUNCH_CHECK("k_pass_flags");
        b = tmp_bytes;
        BFS_CUDA(cub::DeviceScan::InclusiveSum(tmp, b, flags, scan, static_cast<int>(n), s));
        k_pass_scatter<<<bl, th, 0, s>>>(v_out, scan, n, gid);
        BFS_LAUNCH_CHECK("k_pass_scatter");
    }
    BFS_CUDA(cudaMemcpyAsync(d_perm, v_out, sizeof(int) * n, cudaMemcpyDeviceToDevice, s));
    k_offsets<<<bl, th, 0, s>>>(flags, scan, n, d_offsets);
    BFS_LAUNCH_CHECK("k_offsets");
    unsigned ng = 0;
    BFS_CUDA(cudaMemcpyAsync(&ng, scan + (n - 1), sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    BFS_CUDA(cudaStreamSynchronize(s));
    // delegates in group order, then sorted by (mt, group)
    int* dl_group;
    BFS_TRY(sc.alloc(reinterpret_cast<void**>(&dl_group), sizeof(int) * ng));
    k_select_delegates<<<ng, kDelegateLanes, 0, s>>>(d_cands, d_perm, n, d_offsets, dl_group);
    BFS_LAUNCH_CHECK("k_select_delegates");
    const int blg = static_cast<int>((ng + th - 1) / th);
    k_delegate_keys<<<blg, th, 0, s>>>(d_cands, dl_group, ng, k_in, v_in);
    BFS_LAUNCH_CHECK("k_delegate_keys");
    size_t b = tmp_bytes;
    BFS_CUDA(cub::DeviceRadixSort::SortPairs(tmp, b, k_in, k_out, v_in,
                                             reinterpret_cast<unsigned*>(d_delegates),
                                             static_cast<int>(ng), 0, 64, s));
    *h_ngroups = ng;
    return BFS_OK;
}
