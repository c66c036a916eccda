// Test infrastructure only: a C-ABI wrapper around the reference's own
// candidate report (COutChunkHeader::createOutStr / writeReport /
// read_outputlogfile_line, MyVSLib_C++/OutChunkHeader.cpp:89-227), compiled
// with that unchanged source by oracle/Makefile into
// oracle/_ref/libref_report.so.  Nothing in the product links it.
#include <vector>

#include "OutChunkHeader.h"

extern "C" {

// n records; ints[9*i..] = {nrows, ncols, suc_row, suc_col, width, block, chunk, 0, 0}
void ref_write_report(const char* path, int n, const int* ints, const float* snr, const float* cohdisp,
                      float pulse_length) {
    std::vector<COutChunkHeader> v;
    for (int i = 0; i < n; ++i) {
        const int* a = ints + 9 * i;
        v.emplace_back(a[0], a[1], a[2], a[3], a[4], snr[i], cohdisp[i], a[5], a[6]);
    }
    COutChunkHeader::writeReport(path, &v, pulse_length);
}

// out ints: block, chunk, rows, cols, suc_row, suc_col, width; floats: cohdisp, snr
int ref_read_report_line(const char* path, int line, int* ints, float* floats) {
    return COutChunkHeader::read_outputlogfile_line(path, line, ints, ints + 1, ints + 2, ints + 3, ints + 4,
                                                    ints + 5, ints + 6, floats, floats + 1) ? 1 : 0;
}

}  // extern "C"
