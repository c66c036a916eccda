// Square cut-outs of a DM-time plane around a detection, for vetting
// (CFragment; the reference's CChunkB::cutQuadraticFragment,
// MyVSLib_C++/CDMT/ChunkB.cpp:255-275).  The rule is the reference's: with
// rows < cols the fragment is the rows x rows block of all rows starting at
// column (target_col / rows) * rows; otherwise the cols x cols block at the
// top of the plane.  The reference copies each fragment row with one memcpy
// from the row-major plane, so where a block runs past the right edge it
// continues into the next row; the kernel reads the same flat positions and
// gives 0 past the end of the plane (where the reference would read outside
// its array).
#include <cuda_runtime.h>

#include "internal.h"

namespace {

__global__ void k_cut_fragment(const float* __restrict__ plane, long long total, int cols, int dim,
                               long long start, float* __restrict__ out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (j >= dim) return;
    const long long flat = static_cast<long long>(i) * cols + start + j;
    out[static_cast<size_t>(i) * dim + j] = flat < total ? __ldg(plane + flat) : 0.0f;
}

}  // namespace

using namespace bfs;

extern "C" bfs_status bfs_cut_fragment(const float* d_plane, int rows, int cols, int target_row,
                                       int target_col, float* d_out, int* row_begin, int* col_begin,
                                       int* dim, void* stream) {
    BFS_ARG(rows >= 1 && cols >= 1, "bad plane shape %dx%d", rows, cols);
    BFS_ARG(target_row >= 0 && target_row < rows && target_col >= 0 && target_col < cols,
            "target (%d, %d) outside the plane", target_row, target_col);
    int rb, cb, d;
    long long start;
    if (rows < cols) {
        d = rows;
        cb = (target_col / rows) * rows;
        rb = 0;
        start = cb;
    } else {
        d = cols;
        const int part = target_row / rows;  // the reference's block index (0 for any row)
        rb = part;
        cb = 0;
        start = static_cast<long long>(part) * cols;
    }
    if (row_begin) *row_begin = rb;
    if (col_begin) *col_begin = cb;
    if (dim) *dim = d;
    if (!d_out) return BFS_OK;
    BFS_ARG(d_plane != nullptr, "null plane");
    BFS_ARG(d <= 65535, "fragment dimension %d too large for this build", d);
    dim3 grid((d + 255) / 256, d);
    k_cut_fragment<<<grid, 256, 0, as_stream(stream)>>>(d_plane, static_cast<long long>(rows) * cols, cols, d,
                                                         start, d_out);
    BFS_LAUNCH_CHECK("k_cut_fragment");
    return BFS_OK;
}
