// Test infrastructure only: a C-ABI wrapper around the reference's own CPU
// implementation of the Pravir-style FDMT (FDMT / FDMTCPU,
// MyVSLib_C++/FDMT_PRAVIR/fdmt_base.cpp, fdmt_cpu.cpp, fdmtUtils.cpp),
// compiled together with those unchanged sources by oracle/Makefile into
// oracle/_ref/libref_pravir.so.  Nothing in the product links it.
// FDMTCPU::execute prints a timing line to stdout; the wrapper silences
// stdout at the file-descriptor level for the call.
#include <cstdio>
#include <exception>
#include <unistd.h>
#include <fcntl.h>
#include <omp.h>

#include "fdmt_cpu.hpp"

namespace {
struct Quiet {
    int saved = -1;
    Quiet() { fflush(stdout); saved = dup(1); int n = open("/dev/null", O_WRONLY); if (n >= 0) { dup2(n, 1); close(n); } }
    ~Quiet() { fflush(stdout); if (saved >= 0) { dup2(saved, 1); close(saved); } }
};
}  // namespace

extern "C" {

// Output rows (length of the final dt grid), or -1 if the reference throws.
long ref_pravir_rows(float fmin, float fmax, long nchans, long nsamps, float tsamp, long dt_max,
                     long dt_step, long dt_min) {
    try {
        Quiet q;
        FDMTCPU f(fmin, fmax, nchans, nsamps, tsamp, dt_max, dt_step, dt_min);
        return static_cast<long>(f.get_dt_grid_final().size());
    } catch (const std::exception&) {
        return -1;
    }
}

// Final dt grid into dt (cap entries); returns its length or -1.
long ref_pravir_dt_grid(float fmin, float fmax, long nchans, long nsamps, float tsamp, long dt_max,
                        long dt_step, long dt_min, long* dt, long cap) {
    try {
        Quiet q;
        FDMTCPU f(fmin, fmax, nchans, nsamps, tsamp, dt_max, dt_step, dt_min);
        const auto& g = f.get_dt_grid_final();
        for (size_t i = 0; i < g.size() && static_cast<long>(i) < cap; ++i) dt[i] = static_cast<long>(g[i]);
        return static_cast<long>(g.size());
    } catch (const std::exception&) {
        return -1;
    }
}

// A fresh FDMTCPU(...).execute(in, out) with `threads` OpenMP threads (its
// loops are independent per sub-band / per output row, so the result does
// not depend on the thread count).  Returns 0, or -1 if the reference throws.
int ref_pravir_execute(float fmin, float fmax, long nchans, long nsamps, float tsamp, long dt_max,
                       long dt_step, long dt_min, const float* in, float* out, long out_size,
                       int threads) {
    try {
        Quiet q;
        omp_set_num_threads(threads > 0 ? threads : 1);
        FDMTCPU f(fmin, fmax, nchans, nsamps, tsamp, dt_max, dt_step, dt_min);
        f.execute(in, static_cast<size_t>(nchans * nsamps), out, static_cast<size_t>(out_size));
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

}  // extern "C"
