// Test infrastructure only: a C-ABI wrapper around the reference's own CPU
// FDMT class (CFdmtCpu, MyVSLib_C++/FDMT/FdmtCpu.cpp) so the parity tests and
// the CPU-baseline leg of bench.py can call it through ctypes.  This file is
// compiled together with the reference sources (unchanged) by oracle/Makefile
// into oracle/_ref/libref_fdmt.so.  Nothing in the product links it.
//
// The reference prints "NUmOperation = ..." to stdout on every
// process_image call (FdmtCpu.cpp:228); the wrapper silences stdout at the file
// descriptor level for the duration of the call so a caller's own stdout
// protocol (one JSON line) stays clean.
#include <cstdio>
#include <cstring>
#include <unistd.h>
#include <fcntl.h>
#include <omp.h>

#include "FdmtCpu.h"

namespace {
struct StdoutSilencer {
    int saved = -1;
    StdoutSilencer() {
        fflush(stdout);
        saved = dup(1);
        int devnull = open("/dev/null", O_WRONLY);
        if (devnull >= 0) { dup2(devnull, 1); close(devnull); }
    }
    ~StdoutSilencer() {
        fflush(stdout);
        if (saved >= 0) { dup2(saved, 1); close(saved); }
    }
};
}  // namespace

extern "C" {

// Runs CFdmtCpu(fmin, fmax, nchan, cols, max_dt).process_image(in, out, b_ones)
// with `threads` OpenMP threads.  Returns the number of FDMT iterations.
// NOTE: the reference's level-0 initialisation (FdmtCpu.cpp:352-366) runs a
// loop-carried recurrence over delay rows under `omp parallel for`; with more
// than one thread its result depends on thread timing.  Parity comparisons
// therefore use threads == 1; timing runs may use all cores.
int ref_fdmt_cpu_process(float fmin, float fmax, int nchan, int cols, int max_dt,
                         float* in, float* out, int b_ones, int threads) {
    omp_set_num_threads(threads > 0 ? threads : 1);
    StdoutSilencer quiet;
    CFdmtCpu fdmt(fmin, fmax, nchan, cols, max_dt);
    fdmt.process_image(in, out, b_ones != 0);
    return fdmt.m_iNumIter;
}

// Plan introspection: number of iterations, then per level the number of
// sub-bands and the row cumsum table (m_pparrRowsCumSum_h).
int ref_fdmt_cpu_plan(float fmin, float fmax, int nchan, int cols, int max_dt,
                      int* quant_mtrx, int* cumsum_flat, int cumsum_cap) {
    StdoutSilencer quiet;
    CFdmtCpu fdmt(fmin, fmax, nchan, cols, max_dt);
    int pos = 0;
    for (int i = 0; i <= fdmt.m_iNumIter; ++i) {
        quant_mtrx[i] = fdmt.m_parrQuantMtrx_h[i];
        for (int k = 0; k <= fdmt.m_parrQuantMtrx_h[i]; ++k) {
            if (pos < cumsum_cap) cumsum_flat[pos] = fdmt.m_pparrRowsCumSum_h[i][k];
            ++pos;
        }
    }
    return fdmt.m_iNumIter;
}

}  // extern "C"
