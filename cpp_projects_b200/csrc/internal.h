// Internal helpers shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <string>
#include <vector>

#include "bfs.h"

namespace bfs {

// Thread-local last-error message (bfs_last_error()).
void set_error(const char* fmt, ...);
bfs_status fail(bfs_status st, const char* fmt, ...);

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// cudaMallocAsync from the device's default pool, which keeps freed memory.
bfs_status stream_alloc(void** p, size_t bytes, cudaStream_t s);

#define BFS_CUDA(call)                                                                     \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return ::bfs::fail(BFS_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call,     \
                               cudaGetErrorString(e_));                                    \
    } while (0)

#define BFS_LAUNCH_CHECK(what)                                                             \
    do {                                                                                   \
        cudaError_t e_ = cudaGetLastError();                                               \
        if (e_ != cudaSuccess)                                                             \
            return ::bfs::fail(BFS_ERR_CUDA, "launch of %s failed: %s", what,              \
                               cudaGetErrorString(e_));                                    \
    } while (0)

#define BFS_ARG(cond, ...)                                                                 \
    do {                                                                                   \
        if (!(cond)) return ::bfs::fail(BFS_ERR_ARG, __VA_ARGS__);                         \
    } while (0)

// ---------------------------------------------------------------------------
// FDMT plan (host side).  Built once per (fmin, fmax, nchan, ncols, max_dt).
// ---------------------------------------------------------------------------
struct FdmtLevel {
    int nsub = 0;                 // sub-bands at this level
    std::vector<int> rows;        // rows per sub-band
    std::vector<int> cum;         // nsub + 1 cumulative rows
    std::vector<float> freq;      // nsub + 1 sub-band edges (MHz)
    // level >= 1: one entry per output row (global indices in the previous plane)
    std::vector<int> a_row, b_row, shift;
    // maximum look-back (samples) of any row of this level, counting level 0
    std::vector<int> lookback;    // per row
    int total_rows() const { return cum.empty() ? 0 : cum[nsub]; }
};

struct FdmtPlanHost {
    int kind = BFS_PLAN_KEITH;
    float fmin = 0, fmax = 0;
    int nchan = 0, ncols = 0, max_dt = 0;
    int niter = 0;
    int rows_per_chan0 = 0;  // level-0 rows of every channel (d0 + 1); Pravir plans: 0
                             // (per channel: lv[0].rows, delays dt0)
    std::vector<int> dt0;    // Pravir plans: the delay of every level-0 row
    std::vector<int> dt_out; // delay of every output row
    std::vector<FdmtLevel> lv;  // niter + 1 levels
    int out_rows() const { return lv.empty() ? 0 : lv.back().total_rows(); }
};

// Builds the plan exactly as the reference's CFdmtB/CFdmtCpu do.  Returns
// BFS_OK or BFS_ERR_ARG (with the message set).
bfs_status build_fdmt_plan(float fmin, float fmax, int nchan, int ncols, int max_dt,
                           FdmtPlanHost* out);
// The reference's second FDMT variant (FDMT_PRAVIR): delay grids dt_min ..
// dt_max step dt_step per sub-band, window-mean level 0, rounded mid-band
// mappings.  BFS_ERR_ARG where the reference throws.
bfs_status build_pravir_plan(float fmin, float fmax, int nchan, int ncols, int dt_max, int dt_step,
                             int dt_min, FdmtPlanHost* out);

// Inverse row tables of the adjoint: for level l >= 1 and every row i of the
// level-(l-1) plane, the level-l rows g that read row i, with the shift of
// the read (0 as the tail row a_g, s_g as the head row b_g), in ascending g.
struct AdjointTables {
    std::vector<size_t> off_pos;  // per level: start of its nrows+1 offsets in `off`
    std::vector<size_t> ent_pos;  // per level: start of its entries in `ent`
    std::vector<int> off;         // CSR offsets (relative to the level's entries)
    std::vector<int> ent;         // pairs {g, shift}
    bool built = false;
};
void build_adjoint_tables(const FdmtPlanHost& p, AdjointTables* out);

// FDMT of 0/1 rows: every level-0 value of a 0/1 row is exactly 0 or 1 and
// every merge adds integers, so output row d at sample t is exactly the
// number of channels c with weight 1 whose total delay along the merge tree,
// tau(d, c) (the level-0 row plus every head shift on the path), is <= t.
// tau is row-major [out_row][channel]; max_tau its largest value.
void build_ones_delays(const FdmtPlanHost& p, std::vector<int>* tau, int* max_tau);

// ---------------------------------------------------------------------------
// Fused "head" of the FDMT: levels 0..k of one group of 2^k adjacent channels
// computed by one CTA over a time tile, all intermediate levels in shared
// memory.  Tables index rows local to the group's shared-memory planes.
// ---------------------------------------------------------------------------
constexpr int kHeadMaxDepth = 8;

struct HeadGroup {                  // device-side, one per channel group
    int halo;                       // samples of look-back of the group's level-k rows
    int out_row0;                   // first row of the group's sub-band in the level-k plane
    int rows[kHeadMaxDepth + 1];    // rows of the group at levels 0..k
    int tab_off[kHeadMaxDepth + 1]; // offset of level l's table (l >= 1)
};

struct HeadPlan {
    int depth = 0;          // k (0 = no fused head)
    int group = 1;          // 2^k channels per CTA
    int tile = 0;           // output samples per CTA
    int width = 0;          // tile + max halo, rounded to a warp: threads per CTA
    int rows_a = 0;         // shared rows of the even-level buffer (level 0, 2, ...)
    int rows_b = 0;         // shared rows of the odd-level buffer (>= group: it first
                            // stages the group's input rows)
    int tab_rows = 0;       // largest per-group table (levels 1..k), staged in shared memory
    size_t smem_bytes = 0;
    std::vector<HeadGroup> groups;
    std::vector<int> tab;   // 4 ints per row: {a_local, b_local, shift, 0}
};

// Head plan for depth k and tile width; returns false when k is not usable
// (k > trailing zero bits of nchan, k > niter, or too much shared memory).
bool build_head_plan(const FdmtPlanHost& p, int k, int tile, size_t smem_limit, HeadPlan* out);

// ---------------------------------------------------------------------------
// Fused merge segment: levels l0+1..l1 in one pass over HBM.  The level-l1
// plane is cut into tiles of `rows` consecutive rows x `tile` samples.  For
// one such tile the rows of levels l0..l1-1 it depends on (a row DAG through
// the merge tables) are held in shared memory, each over its own window of
// samples: a row reached from the tile's rows through head shifts between
// lo and hi samples in total needs the samples [t0 - hi, t0 + tile - lo),
// which is `tile` + (hi - lo) columns wide, and hi - lo stays small (the
// shifts of neighbouring rows differ by a sample or two), however large the
// shifts themselves are.  So any adjacent levels fuse, the last ones
// included, with only the level-l0 rows read from HBM and the level-l1
// rows written.
// ---------------------------------------------------------------------------
constexpr int kSegMaxLevels = 6;
constexpr int kSegTile = 256;    // output samples per segment tile
constexpr int kSegMaxChunks = 12;  // 32-column chunks per shared row at most

struct SegTile {                 // device-side, one per row tile of a segment
    int ent;                     // first entry of the tile in the segment's entries
    int n[kSegMaxLevels + 1];    // n[0] input rows, n[i] rows of level l0 + i (n[m]: output)
};

// Shared memory: three buffers X0, Y, X1, each of its rows, then a row of
// -0.0 (x + -0 == x bit for bit: the head row of rows without one) and a
// guard row (a chunk of the last row may read up to one pitch past it, in
// columns no written sample depends on); then the entries of two tiles.
// Level i of a tile is held in X (i even) or Y (i odd); a CTA runs tiles one
// after another, loading the next tile's input rows into the other X buffer
// while it merges the current one.  Entries, 4 ints each, in the tile's
// order: n[0] input rows {plane row, window lead E (a multiple of 4, so each
// row's window starts on a 16-byte boundary of the plane), 0, offset in X},
// then for every level i = 1..m its rows {offset of the tail row's sample and
// of the head row's sample minus the shift, both in the buffer of level
// i-1, first sample that adds the head row relative to t0 (shift + lead),
// destination: offset in the buffer of level i, or the plane row at level
// m}.  Offsets count floats; local column u of a row with lead E holds
// sample t0 - E + u.
struct SegPlan {
    int l0 = 0, l1 = 0;
    int rows = 0;                // output rows per tile
    int tile = 0;                // output samples per tile (multiple of 32)
    int nc = 0;                  // 32-column chunks per shared row
    int pitch = 0;               // floats per shared row (32 nc)
    int rows_x = 0, rows_y = 0;  // rows of buffer X (levels l0, l0+2, ..) and Y (l0+1, ..)
    int size_x = 0, size_y = 0;  // floats of a buffer: its rows, the -0.0 row, the guard row
    int max_thr = 0;             // tiles with t0 >= max_thr never need the t >= shift test
    int threads = 0;             // CTA size of its kernel (0: 256 when two CTAs fit an SM, else 512)
    bool single = false;         // one input buffer: the next tile loads after this one is merged
    int r0c = 0;                 // input segment (levels 1..l1 straight from the channels):
                                 // level-0 rows per channel; 0 = the input is a level plane
    int max_in_rows = 0;         // most input rows of one tile
    int64_t in_rows = 0;         // input rows summed over tiles (HBM reads per time tile)
    int y0 = 0, x1 = 0;          // offsets of buffers Y and X1 (X0 is at 0)
    int ent_base = 0;            // offset (floats) of the two staged entry buffers
    int max_ent = 0;             // most entries of one tile
    size_t smem_bytes = 0;
    std::vector<SegTile> tiles;
    std::vector<int> ent;
};

// Input segment (from_input, BFS_PLAN_KEITH, l0 = 0): the tile's input rows
// are channels of the filterbank, each over the window its level-0 rows need
// (r more samples on the left for the running mean of row r), and level 1
// is formed straight from them: a level-1 entry's w packs the destination
// (low 20 bits), the tail and head rows' level-0 row numbers (4 bits each at
// 20 and 24) and the shift (4 bits at 28); its x / y point at sample t of the
// tail channel and t - shift of the head channel.  No level-0 plane exists.
//
// Segment plan for levels l0+1..l1 with `rows` output rows and `tile`
// samples per tile; false when it needs more than kSegMaxLevels levels,
// kSegMaxChunks chunks per row or smem_limit bytes of shared memory (or, for
// an input segment, a level-0 depth, shift or offset beyond its packing).
bool build_seg_plan(const FdmtPlanHost& p, int l0, int l1, int rows, int tile, size_t smem_limit,
                    SegPlan* out, bool from_input = false, bool single = false);

}  // namespace bfs
