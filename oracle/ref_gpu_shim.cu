// Test / measurement infrastructure only: a C-ABI wrapper around the
// reference's OWN GPU classes, compiled (by oracle/Makefile) together with the
// unchanged reference sources into oracle/_ref/libref_gpu.so:
//   CFdmtGpu                MyVSLib_C++/FDMT/FdmtGpu.cu (+ FdmtCpu.cpp, FdmtB.cpp)
//   clusterization::*       MyVSLib_C++/Clusterization/Clusterization.cu
//                           (+ select_delegates.cu, Segmented_sort.cu)
// It provides the "plain per-chunk GPU form" the reference itself runs, for
// timing and as a second parity check.  Nothing in the product links it.
#include <cstdio>
#include <cstring>
#include <string>
#include <unistd.h>
#include <fcntl.h>

#include "Clusterization.cuh"
#include "FdmtGpu.cuh"

namespace {
struct Quiet {
    int saved = -1;
    Quiet() { fflush(stdout); saved = dup(1); int n = open("/dev/null", O_WRONLY); if (n >= 0) { dup2(n, 1); close(n); } }
    ~Quiet() { fflush(stdout); if (saved >= 0) { dup2(saved, 1); close(saved); } }
};
}  // namespace

extern "C" {

void* ref_fdmt_gpu_create(float fmin, float fmax, int nchan, int cols, int max_dt) {
    Quiet q;
    return new CFdmtGpu(fmin, fmax, nchan, cols, max_dt);
}

void ref_fdmt_gpu_destroy(void* h) {
    Quiet q;  // the reference's code prints a line here
    delete static_cast<CFdmtGpu*>(h);
}

// d_in, d_out: device pointers; runs on the default stream (as the reference does).
int ref_fdmt_gpu_process(void* h, float* d_in, float* d_out, int b_ones) {
    static_cast<CFdmtGpu*>(h)->process_image(d_in, d_out, b_ones != 0);
    return static_cast<int>(cudaGetLastError());
}

// The heap gather (widths 1..W) into host memory; returns the candidate count.
unsigned ref_gather_heap(const float* d_plane, int rows, int cols, const float* d_thr, int W,
                         void* h_out, unsigned cap) {
    Cand* d_c = nullptr;
    unsigned n = 0;
    clusterization::gather_candidates_in_heap_with_plan(d_plane, rows, cols, *d_thr, W, &d_c, &n);
    if (d_c && h_out && n) cudaMemcpy(h_out, d_c, sizeof(Cand) * (n < cap ? n : cap), cudaMemcpyDeviceToHost);
    if (d_c) cudaFree(d_c);
    return n;
}

// The dynamic gather (widths 1..2^Q); candidates in the reference's atomic order.
unsigned ref_gather_dynamic(const float* d_plane, int rows, int cols, const float* d_thr, int Q,
                            void* h_out, unsigned cap) {
    Cand* d_c = nullptr;
    unsigned n = 0;
    clusterization::gather_candidates_in_dynamicalArray(d_plane, rows, cols, *d_thr, Q, &d_c, &n);
    cudaDeviceSynchronize();
    if (d_c && h_out && n) cudaMemcpy(h_out, d_c, sizeof(Cand) * (n < cap ? n : cap), cudaMemcpyDeviceToHost);
    if (d_c) cudaFree(d_c);
    return n;
}

// The body of clusterization_main (Clusterization.cu:17-54): heap gather
// (widths 1..W) + complete_clusterization with its log.  The reference's
// function itself falls off its end without a return on the success path
// (undefined behaviour that corrupted the host stack here), so its two calls
// are made directly.  Returns the candidate count.
unsigned ref_cluster_heap(const float* d_plane, int rows, int cols, const float* d_thr, int W,
                          const int* d_metrics, const char* logfile, float delt_bin, float t0) {
    Quiet q;
    Cand* d_c = nullptr;
    unsigned n = 0;
    clusterization::gather_candidates_in_heap_with_plan(d_plane, rows, cols, *d_thr, W, &d_c, &n);
    if (n > 0)
        clusterization::complete_clusterization(d_c, n, d_metrics, std::string(logfile), delt_bin, t0, true);
    cudaDeviceSynchronize();
    if (d_c) cudaFree(d_c);
    return n;
}

// gather_candidates_in_dynamicalArray (widths 1..2^Q) + complete_clusterization
// (log written to `logfile`); returns the candidate count.
unsigned ref_search_dynamic(const float* d_plane, int rows, int cols, const float* d_thr, int Q,
                            const int* d_metrics, const char* logfile, float delt_bin, float t0) {
    Quiet q;
    Cand* d_c = nullptr;
    unsigned n = 0;
    clusterization::gather_candidates_in_dynamicalArray(d_plane, rows, cols, *d_thr, Q, &d_c, &n);
    if (n > 0)
        clusterization::complete_clusterization(d_c, n, d_metrics, std::string(logfile), delt_bin, t0, true);
    cudaDeviceSynchronize();
    if (d_c) cudaFree(d_c);
    return n;
}

}  // extern "C"
