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

// Pass key: (group id << fbits) | (field - fmin), in 32 bits when it fits.
template <typename K>
__global__ void k_pass_keys(const bfs_cand* __restrict__ c, const unsigned* __restrict__ gid,
                            unsigned n, int field, int fmin, int fbits, K* __restrict__ keys,
                            unsigned* __restrict__ vals) {
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const K g = gid ? static_cast<K>(gid[i]) : K(0);
    const K f = static_cast<K>(static_cast<unsigned>(
        static_cast<long long>(field_of(c[i], field)) - static_cast<long long>(fmin)));
    keys[i] = (fbits >= static_cast<int>(8 * sizeof(K)) ? K(0) : (g << fbits)) | f;
    vals[i] = i;
}

// Group starts in the sorted order: the group changes, or the field grows by
// more than the metric.  A key's low fbits bits are its field minus the
// smallest field (exact: fbits covers the range), so the sorted keys alone
// give both tests.
template <typename K>
__global__ void k_pass_flags(const K* __restrict__ keys, unsigned n, int fbits, long long metric,
                             unsigned* __restrict__ flags) {
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    unsigned f = 1u;
    if (i > 0) {
        const bool whole = fbits >= static_cast<int>(8 * sizeof(K));
        const K k0 = keys[i - 1], k1 = keys[i];
        const K g0 = whole ? K(0) : (k0 >> fbits);
        const K g1 = whole ? K(0) : (k1 >> fbits);
        if (g0 == g1) {
            const K mask = whole ? ~K(0) : ((K(1) << fbits) - K(1));
            const long long d = static_cast<long long>(k1 & mask) - static_cast<long long>(k0 & mask);
            f = (d > metric) ? 1u : 0u;
        }
    }
    flags[i] = f;
}

// Range of each field (biased so signed order is unsigned order).
__global__ void k_field_range(const bfs_cand* __restrict__ c, unsigned n, unsigned* __restrict__ r) {
    unsigned lo[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, hi[3] = {0u, 0u, 0u};
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const bfs_cand v = c[i];
        const unsigned f[3] = {biased(v.mt), biased(v.mdt), biased(v.mwidth)};
        for (int k = 0; k < 3; ++k) { lo[k] = min(lo[k], f[k]); hi[k] = max(hi[k], f[k]); }
    }
    for (int k = 0; k < 3; ++k) {
        for (int o = 16; o > 0; o >>= 1) {
            lo[k] = min(lo[k], __shfl_down_sync(0xffffffffu, lo[k], o));
            hi[k] = max(hi[k], __shfl_down_sync(0xffffffffu, hi[k], o));
        }
        if ((threadIdx.x & 31) == 0) { atomicMin(r + 2 * k, lo[k]); atomicMax(r + 2 * k + 1, hi[k]); }
    }
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

// Delegate selection, exactly the reference's select_delegates_kernel
// (64 lanes per group; lane l keeps the first strict maximum of msnr among the
// group positions l, l+64, ...; a tree reduction `take lane l+s if strictly
// greater` for s = 32..1) but split in two so that groups of millions of
// members do not serialise on 64 threads:
//   k_delegate_lanes  every position of every group, 16 per thread (stride 64,
//                     so a thread stays on one lane of a group) keeps the
//                     largest key (ordered msnr << 32 | ~position) and folds it
//                     into its (group, lane) slot with a 64-bit atomicMax:
//                     the largest value, earliest position on ties = the
//                     reference lane's strided scan;
//   k_delegate_tree   one 64-thread block per group runs the reference's tree.
constexpr int kLanePositions = 16;
constexpr int kLaneThreads = 256;
constexpr int kLaneBlockSpan = kLaneThreads * kLanePositions;  // positions per block

__device__ __forceinline__ unsigned ordered_bits(float f) {
    const unsigned b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__device__ __forceinline__ int group_of(const int* __restrict__ offsets, int ngroups, int i) {
    int lo = 0, hi = ngroups - 1;  // largest g with offsets[g] <= i
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(offsets + mid) <= i) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__global__ void __launch_bounds__(kLaneThreads)
k_delegate_lanes(const bfs_cand* __restrict__ c, const int* __restrict__ perm, int n,
                 const int* __restrict__ offsets, int ngroups,
                 unsigned long long* __restrict__ slots) {
    const int sub = threadIdx.x / kDelegateLanes, lane = threadIdx.x % kDelegateLanes;
    const int base = blockIdx.x * kLaneBlockSpan + sub * (kDelegateLanes * kLanePositions) + lane;
    int g = -1, g_beg = 0, g_end = 0;
    unsigned long long best = 0ull;
    for (int k = 0; k < kLanePositions; ++k) {
        const int i = base + k * kDelegateLanes;
        if (i >= n) break;
        if (g < 0 || i >= g_end) {
            if (best) atomicMax(slots + static_cast<size_t>(g) * kDelegateLanes + ((base - g_beg) & 63), best);
            g = group_of(offsets, ngroups, i);
            g_beg = __ldg(offsets + g);
            g_end = __ldg(offsets + g + 1);
            best = 0ull;
        }
        const unsigned pos = static_cast<unsigned>(i - g_beg);
        const unsigned long long key =
            (static_cast<unsigned long long>(ordered_bits(c[__ldg(perm + i)].msnr)) << 32) |
            static_cast<unsigned long long>(0xffffffffu - pos);
        best = key > best ? key : best;
    }
    if (best) atomicMax(slots + static_cast<size_t>(g) * kDelegateLanes + ((base - g_beg) & 63), best);
}

__global__ void __launch_bounds__(kDelegateLanes)
k_delegate_tree(const bfs_cand* __restrict__ c, const int* __restrict__ perm,
                const int* __restrict__ offsets, const unsigned long long* __restrict__ slots,
                int* __restrict__ delegates) {
    __shared__ float sv[kDelegateLanes];
    __shared__ int si[kDelegateLanes];
    const int g = blockIdx.x;
    const int beg = offsets[g];
    const int len = offsets[g + 1] - beg;
    const int lane = threadIdx.x;
    float v = -FLT_MAX;
    int idx = lane;  // the reference leaves the lane id in idle lanes
    if (lane < len) {
        const unsigned long long key = slots[static_cast<size_t>(g) * kDelegateLanes + lane];
        const unsigned pos = 0xffffffffu - static_cast<unsigned>(key & 0xffffffffull);
        idx = perm[beg + pos];
        v = c[idx].msnr;
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

bfs_status launch_select_delegates(const bfs_cand* c, const int* perm, unsigned n,
                                   const int* offsets, unsigned ngroups, int* out,
                                   unsigned long long* slots, cudaStream_t s) {
    if (ngroups == 0) return BFS_OK;
    BFS_CUDA(cudaMemsetAsync(slots, 0, sizeof(unsigned long long) * kDelegateLanes * ngroups, s));
    const int blocks = static_cast<int>((n + kLaneBlockSpan - 1) / kLaneBlockSpan);
    k_delegate_lanes<<<blocks, kLaneThreads, 0, s>>>(c, perm, static_cast<int>(n), offsets,
                                                     static_cast<int>(ngroups), slots);
    BFS_LAUNCH_CHECK("k_delegate_lanes");
    k_delegate_tree<<<ngroups, kDelegateLanes, 0, s>>>(c, perm, offsets, slots, out);
    BFS_LAUNCH_CHECK("k_delegate_tree");
    return BFS_OK;
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
        bfs_status st = stream_alloc(p, bytes, s);
        if (st != BFS_OK) return st;
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
    BFS_ARG(n > 0 && n < 0x7fffffffu, "bad candidate count %u", n);
    cudaStream_t s = as_stream(stream);
    Scratch sc{s, {}};
    unsigned long long* slots;
    BFS_TRY(sc.alloc(reinterpret_cast<void**>(&slots),
                     sizeof(unsigned long long) * kDelegateLanes * ngroups));
    return launch_select_delegates(d_cands, d_perm, n, d_offsets, ngroups, d_delegates, slots, s);
}

static int bits_for(unsigned long long v) {
    int b = 0;
    while (b < 64 && (v >> b) != 0ull) ++b;
    return b;
}

// One pass of the split: sort by (group, field), flag the positions where the
// group changes or the field jumps by more than the metric, and renumber the
// groups.  With sort_only the pass cannot split (the metric is at least the
// field's whole range): the sort alone fixes the member order, the groups and
// their boundaries stay those of the previous pass.
template <typename K>
static bfs_status cluster_pass(const bfs_cand* d_cands, unsigned n, int field, int fmin, int fbits,
                               int end_bit, long long metric, unsigned* gid, bool first, void* kin,
                               void* kout, unsigned* v_in, unsigned* v_out, unsigned* flags,
                               unsigned* scan, void* tmp, size_t tmp_bytes, cudaStream_t s,
                               bool sort_only = false) {
    const int th = 256;
    const int bl = static_cast<int>((n + th - 1) / th);
    K* k_in = static_cast<K*>(kin);
    K* k_out = static_cast<K*>(kout);
    k_pass_keys<K><<<bl, th, 0, s>>>(d_cands, first ? nullptr : gid, n, field, fmin, fbits, k_in, v_in);
    BFS_LAUNCH_CHECK("k_pass_keys");
    size_t b = tmp_bytes;
    BFS_CUDA(cub::DeviceRadixSort::SortPairs(tmp, b, k_in, k_out, v_in, v_out, static_cast<int>(n),
                                             0, end_bit > 0 ? end_bit : 1, s));
    if (sort_only) return BFS_OK;
    k_pass_flags<K><<<bl, th, 0, s>>>(k_out, n, fbits, metric, flags);
    BFS_LAUNCH_CHECK("k_pass_flags");
    b = tmp_bytes;
    BFS_CUDA(cub::DeviceScan::InclusiveSum(tmp, b, flags, scan, static_cast<int>(n), s));
    k_pass_scatter<<<bl, th, 0, s>>>(v_out, scan, n, gid);
    BFS_LAUNCH_CHECK("k_pass_scatter");
    return BFS_OK;
}

extern "C" bfs_status bfs_cluster(const bfs_cand* d_cands, uint32_t n, const int* metrics,
                                  int* d_perm, int* d_offsets, int* d_delegates,
                                  uint32_t* h_ngroups, void* stream) {
    return bfs_cluster_grouped(d_cands, n, nullptr, 0, metrics, d_perm, d_offsets, d_delegates,
                               h_ngroups, stream);
}

extern "C" bfs_status bfs_cluster_grouped(const bfs_cand* d_cands, uint32_t n, const int* d_group0,
                                          uint32_t ngroups0, const int* metrics, int* d_perm,
                                          int* d_offsets, int* d_delegates, uint32_t* h_ngroups,
                                          void* stream) {
    BFS_ARG(metrics && h_ngroups, "null argument");
    BFS_ARG(d_group0 == nullptr || ngroups0 >= 1, "ngroups0 must be >= 1 with d_group0");
    *h_ngroups = 0;
    if (n == 0) return BFS_OK;
    BFS_ARG(d_cands && d_perm && d_offsets && d_delegates, "null argument");
    BFS_ARG(n < 0x7fffffffu, "too many candidates");
    cudaStream_t s = as_stream(stream);
    Scratch sc{s, {}};
    unsigned long long *k_in, *k_out;
    unsigned *v_in, *v_out, *gid, *flags, *scan, *range;
    BFS_TRY(sc.alloc(reinterpret_cast<void**>(&k_in), sizeof(unsigned long long) * n));
    BFS_TRY(sc.alloc(reinterpret_cast<void**>(&k_out), sizeof(unsigned long long) * n));
    BFS_TRY(sc.alloc(reinterpret_cast<void**>(&v_in), sizeof(unsigned) * n));
    BFS_TRY(sc.alloc(reinterpret_cast<void**>(&v_out), sizeof(unsigned) * n));
    BFS_TRY(sc.alloc(reinterpret_cast<void**>(&gid), sizeof(unsigned) * n));
    BFS_TRY(sc.alloc(reinterpret_cast<void**>(&flags), sizeof(unsigned) * n));
    BFS_TRY(sc.alloc(reinterpret_cast<void**>(&scan), sizeof(unsigned) * n));
    BFS_TRY(sc.alloc(reinterpret_cast<void**>(&range), sizeof(unsigned) * 6));
    size_t sort64 = 0, sort32 = 0, scan_bytes = 0;
    BFS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, sort64, k_in, k_out, v_in, v_out,
                                             static_cast<int>(n), 0, 64, s));
    BFS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, sort32, reinterpret_cast<unsigned*>(k_in),
                                             reinterpret_cast<unsigned*>(k_out), v_in, v_out,
                                             static_cast<int>(n), 0, 32, s));
    BFS_CUDA(cub::DeviceScan::InclusiveSum(nullptr, scan_bytes, flags, scan, static_cast<int>(n), s));
    void* tmp;
    const size_t tmp_bytes = std::max(std::max(sort64, sort32), scan_bytes);
    BFS_TRY(sc.alloc(&tmp, tmp_bytes));
    const int th = 256;
    const int bl = static_cast<int>((n + th - 1) / th);

    // field ranges -> key widths
    unsigned h_range[6];
    {
        const unsigned init[6] = {0xffffffffu, 0u, 0xffffffffu, 0u, 0xffffffffu, 0u};
        BFS_CUDA(cudaMemcpyAsync(range, init, sizeof(init), cudaMemcpyHostToDevice, s));
        k_field_range<<<std::min(bl, 1184), th, 0, s>>>(d_cands, n, range);
        BFS_LAUNCH_CHECK("k_field_range");
        BFS_CUDA(cudaMemcpyAsync(h_range, range, sizeof(h_range), cudaMemcpyDeviceToHost, s));
        BFS_CUDA(cudaStreamSynchronize(s));
    }
    unsigned groups = d_group0 ? ngroups0 : 1u;
    if (d_group0)
        BFS_CUDA(cudaMemcpyAsync(gid, d_group0, sizeof(unsigned) * n, cudaMemcpyDeviceToDevice, s));
    for (int field = 0; field < 3; ++field) {
        const int fmin = static_cast<int>(h_range[2 * field] ^ 0x80000000u);
        const int fmax = static_cast<int>(h_range[2 * field + 1] ^ 0x80000000u);
        const int fbits = bits_for(static_cast<unsigned long long>(
            static_cast<long long>(fmax) - static_cast<long long>(fmin)));
        const int gbits = bits_for(static_cast<unsigned long long>(groups - 1));
        const int end_bit = fbits + gbits;
        // after a pass that numbered the groups, a metric at least the field's
        // whole range (fmax - fmin < 2^fbits) cannot split: sort only
        const bool sort_only = field > 0 && fbits < 62 &&
                               static_cast<long long>(metrics[field]) >= (1LL << fbits);
        bfs_status st;
        if (end_bit <= 32)
            st = cluster_pass<unsigned>(d_cands, n, field, fmin, fbits, end_bit,
                                        static_cast<long long>(metrics[field]), gid,
                                        field == 0 && d_group0 == nullptr,
                                        k_in, k_out, v_in, v_out, flags, scan, tmp, tmp_bytes, s, sort_only);
        else
            st = cluster_pass<unsigned long long>(d_cands, n, field, fmin, fbits, end_bit,
                                                  static_cast<long long>(metrics[field]), gid,
                                                  field == 0 && d_group0 == nullptr, k_in, k_out,
                                                  v_in, v_out, flags, scan,
                                                  tmp, tmp_bytes, s, sort_only);
        if (st != BFS_OK) return st;
        if (sort_only) continue;   // same groups, same boundaries (groups stay in gid order)
        BFS_CUDA(cudaMemcpyAsync(&groups, scan + (n - 1), sizeof(unsigned), cudaMemcpyDeviceToHost, s));
        BFS_CUDA(cudaStreamSynchronize(s));
    }
    BFS_CUDA(cudaMemcpyAsync(d_perm, v_out, sizeof(int) * n, cudaMemcpyDeviceToDevice, s));
    k_offsets<<<bl, th, 0, s>>>(flags, scan, n, d_offsets);
    BFS_LAUNCH_CHECK("k_offsets");
    const unsigned ng = groups;
    // delegates in group order, then sorted by (mt, group)
    int* dl_group;
    unsigned long long* slots;
    BFS_TRY(sc.alloc(reinterpret_cast<void**>(&dl_group), sizeof(int) * ng));
    BFS_TRY(sc.alloc(reinterpret_cast<void**>(&slots), sizeof(unsigned long long) * kDelegateLanes * ng));
    BFS_TRY(launch_select_delegates(d_cands, d_perm, n, d_offsets, ng, dl_group, slots, s));
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
