// Test infrastructure only: a C-ABI wrapper around the reference's own GUPPI
// header reader (CTelescopeHeader::readGuppiHeader,
// MyVSLib_C++/TelescopeHeader.cpp:175-347), compiled together with that
// unchanged source by oracle/Makefile into oracle/_ref/libref_guppi.so.
// Nothing in the product links it.
#include <cstdio>

#include "TelescopeHeader.h"

extern "C" {

// Reads the header of the block starting at byte `offset` of `path` with the
// reference's reader.  Fills the fields and *data_pos (the file position the
// reader leaves: the start of the block's data).  Returns 1 if the reader
// accepted the header, 0 if not, -1 if the file cannot be opened.
int ref_guppi_read_header(const char* path, long offset, int* nbits, float* chan_bw, int* npol,
                          int* directio, float* centfreq, int* nchan, float* obsbw, long long* blocsize,
                          int* telescope, float* tbin, long* data_pos) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return -1;
    std::fseek(f, offset, SEEK_SET);
    bool dio = false;
    EN_telescope tel = GBT;
    const bool ok = CTelescopeHeader::readGuppiHeader(f, nbits, chan_bw, npol, &dio, centfreq, nchan,
                                                      obsbw, blocsize, &tel, tbin);
    *directio = dio ? 1 : 0;
    *telescope = static_cast<int>(tel);
    *data_pos = std::ftell(f);
    std::fclose(f);
    return ok ? 1 : 0;
}

}  // extern "C"
