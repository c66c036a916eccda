// Library self-tests that need the GPU's own arithmetic as the reference.
//
// bfs_selftest_divide: the level-0 kernels divide by small constants with a
// multiply / fused multiply-add split (divide.cuh) instead of __fdiv_rn; the
// FDMT is only bit-exact if that split equals __fdiv_rn for every input.
// This runs the comparison over all 2^32 float bit patterns on the device.
#include <cuda_runtime.h>

#include <cstdint>

#include "divide.cuh"
#include "internal.h"

namespace bfs {
namespace {

constexpr int kSelftestThreads = 256;

__global__ void __launch_bounds__(kSelftestThreads)
k_divide_check(int d, unsigned long long* __restrict__ bad, unsigned* __restrict__ first_bad) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    unsigned long long nbad = 0;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < (1ull << 32);
         i += stride) {
        const unsigned bits = static_cast<unsigned>(i);
        const float x = __uint_as_float(bits);
        const float got = div_small(x, d);
        const float want = __fdiv_rn(x, static_cast<float>(d));
        if (__float_as_uint(got) != __float_as_uint(want)) {
            ++nbad;
            atomicMin(first_bad, bits);
        }
    }
    if (nbad) atomicAdd(bad, nbad);
}

}  // namespace
}  // namespace bfs

using namespace bfs;

extern "C" bfs_status bfs_selftest_divide(int d, uint64_t* mismatches, uint32_t* first_bad,
                                          void* stream) {
    BFS_ARG(mismatches != nullptr, "null argument");
    BFS_ARG(d >= 1, "divisor %d must be positive", d);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    struct Counters {
        unsigned long long bad;
        unsigned first;
    };
    Counters* dc = nullptr;
    BFS_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&dc), sizeof(Counters), s));
    Counters init{0ull, 0xffffffffu};
    cudaError_t e = cudaMemcpyAsync(dc, &init, sizeof(init), cudaMemcpyHostToDevice, s);
    int sms = 148;
    if (e == cudaSuccess) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        k_divide_check<<<sms * 8, kSelftestThreads, 0, s>>>(d, &dc->bad, &dc->first);
        e = cudaGetLastError();
    }
    Counters host{};
    if (e == cudaSuccess) e = cudaMemcpyAsync(&host, dc, sizeof(host), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(dc, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    BFS_CUDA(e);
    *mismatches = host.bad;
    if (first_bad) *first_bad = host.first;
    return BFS_OK;
}
