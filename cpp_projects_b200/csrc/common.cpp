// Error reporting shared by every entry point.
#include <cstdio>
#include <mutex>

#include "internal.h"

namespace bfs {
namespace {
thread_local char g_last_error[1024] = "";
}

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
}

bfs_status fail(bfs_status st, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return st;
}

const char* last_error() { return g_last_error; }

namespace {
std::mutex g_pool_mu;
bool g_pool_ready[64] = {};
}

// Stream-ordered scratch.  The device's default memory pool is told to keep
// freed memory (release threshold = max) so that per-call scratch is recycled
// instead of being unmapped at every stream synchronisation.
bfs_status stream_alloc(void** p, size_t bytes, cudaStream_t s) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(BFS_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev >= 0 && dev < 64) {
        std::lock_guard<std::mutex> lock(g_pool_mu);
        if (!g_pool_ready[dev]) {
            cudaMemPool_t pool;
            if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
                uint64_t keep = UINT64_MAX;
                cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
            }
            cudaGetLastError();
            g_pool_ready[dev] = true;
        }
    }
    e = cudaMallocAsync(p, bytes ? bytes : 16, s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(BFS_ERR_ALLOC, "cudaMallocAsync(%zu): %s", bytes, cudaGetErrorString(e));
    }
    return BFS_OK;
}

}  // namespace bfs

extern "C" const char* bfs_last_error(void) { return bfs::last_error(); }

extern "C" bfs_status bfs_trim_scratch(void) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return bfs::fail(BFS_ERR_CUDA, "cudaGetDevice failed");
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess ||
        cudaMemPoolTrimTo(pool, 0) != cudaSuccess)
        return bfs::fail(BFS_ERR_CUDA, "trimming the device memory pool failed");
    return BFS_OK;
}
extern "C" const char* bfs_version(void) { return "bfs-b200 0.1 (sm_100a)"; }
