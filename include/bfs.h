/* bfs.h — C ABI of the B200-native FRB / pulsar search core.
 *
 * Every entry point is extern "C", takes plain pointers and sizes, returns a
 * bfs_status and never throws.  Unless stated otherwise, pointers named d_*
 * are DEVICE pointers owned by the caller, `stream` is a cudaStream_t passed
 * as void* (NULL = legacy default stream), and work is enqueued
 * asynchronously on that stream.  A plan object is not thread-safe: use one
 * plan per host thread / stream.  bfs_last_error() returns a message for the
 * last failing call on the calling thread.
 *
 * Each declaration names the reference interface it replaces
 * (Iourick/cpp_projects, paths relative to its root, MyVSLib_C++ = "L/").
 */
#ifndef BFS_H
#define BFS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum bfs_status {
    BFS_OK = 0,
    BFS_ERR_ARG = 1,         /* invalid argument / size mismatch                */
    BFS_ERR_CUDA = 2,        /* a CUDA runtime or library call failed           */
    BFS_ERR_OVERFLOW = 3,    /* output capacity exceeded (count still reported) */
    BFS_ERR_TIMEOUT = 4,     /* a bounded device-side wait gave up              */
    BFS_ERR_ALLOC = 5,       /* device or host allocation failed                */
    BFS_ERR_UNSUPPORTED = 6  /* valid request this build does not implement     */
} bfs_status;

/* Candidate record, byte-compatible with the reference's Cand / SCand
 * (L/Clusterization/Candidate.cuh:4-10): 16 bytes. */
typedef struct bfs_cand {
    int mt;      /* start sample of the window          */
    int mdt;     /* row of the DM-time plane (delay)     */
    int mwidth;  /* width code (log2 w or w, see below)  */
    float msnr;  /* window sum / sqrt(w)                 */
} bfs_cand;

const char* bfs_last_error(void);
const char* bfs_version(void);
/* Calls that need temporary device memory take it from the current device's
 * stream-ordered default pool, set to keep freed memory for reuse; this
 * returns the pool's unused memory to the system. */
bfs_status bfs_trim_scratch(void);

/* ------------------------------------------------------------------------
 * FDMT
 * Replaces CFdmtGpu(Fmin, Fmax, nchan, cols, imaxDt) + process_image
 * (L/FDMT/FdmtGpu.cuh:12-53, L/FDMT/FdmtGpu.cu:230-348) whose plan is
 * CFdmtB/CFdmtCpu::create_config (L/FDMT/FdmtB.cpp:141-245,
 * L/FDMT/FdmtCpu.cpp:143-194).
 * Input: nchan x ncols float32, row 0 = fmin channel.  Output: max_dt x ncols,
 * row d = delay d samples across the band.
 * ---------------------------------------------------------------------- */
/* Plan kinds: BFS_PLAN_KEITH — the reference's CFdmtCpu/CFdmtGpu plan
 * (L/FDMT/FdmtB.cpp, FdmtCpu.cpp); BFS_PLAN_PRAVIR — its second FDMT variant
 * (L/FDMT_PRAVIR/fdmt_base.cpp:118-278, fdmt_cpu.cpp:28-301): delay grids
 * dt_min..max_dt step dt_step, window-mean level 0, output rows = the final
 * grid's length (max_dt - dt_min)/dt_step + 1, no fused head. */
enum { BFS_PLAN_KEITH = 0, BFS_PLAN_PRAVIR = 1 };
/* Storage of the FDMT planes between levels (no reference counterpart: the
 * reference is FP32 throughout).  F16 / BF16 store those planes as 16-bit
 * values, row g scaled by 2^-ceil(log2(channels summed into g)); sums are
 * formed in FP32 and the output is FP32.  F32 is the default and the only
 * precision bit-identical to the reference. */
enum { BFS_PREC_F32 = 0, BFS_PREC_F16 = 1, BFS_PREC_BF16 = 2 };
enum { BFS_FDMT_EXTERNAL_WS = 1 };
enum { BFS_FUSE_AUTOTUNE = -2 };

typedef struct bfs_fdmt_desc {
    float fmin;        /* MHz, lower band edge                          */
    float fmax;        /* MHz, upper band edge                          */
    int nchan;         /* input rows (>= 2)                             */
    int ncols;         /* time samples per row (>= 1)                   */
    int max_dt;        /* output rows (>= 1)                            */
    int plan_kind;     /* BFS_PLAN_KEITH                                */
    int precision;     /* BFS_PREC_F32 (default), BFS_PREC_F16, BFS_PREC_BF16 */
    int fuse_depth;    /* BFS_FUSE_AUTOTUNE (-2): measured per shape (cached); -1: deepest
                          head keeping 2 CTAs/SM; 0: level-by-level; k: fuse levels 0..k */
    int flags;         /* BFS_FDMT_EXTERNAL_WS: the plan allocates no planes; use _execute_ws */
    int head_tile;     /* samples per CTA of the fused head (0 = 256)                  */
    int dt_min;        /* BFS_PLAN_PRAVIR: smallest delay of the grid (0)              */
    int dt_step;       /* BFS_PLAN_PRAVIR: grid step (0 is taken as 1)                 */
    float tsamp;       /* BFS_PLAN_PRAVIR: sample time (s), for the DM grid only       */
    int seg_levels;    /* merge levels fused per HBM pass after the head (FP32 plans):
                          0: 3; 1: one pass per level; 2..6                              */
    int seg_rows;      /* output rows per tile of a fused pass (0: the most that keep
                          two CTAs per SM, of 64 / 32 / 16; the autotuner also tries
                          24 and 28, which fit a single-buffered input segment into
                          half an SM's shared memory)                                    */
    int seg_threads;   /* threads per CTA of the fused passes: 256, 512, 1024 (0: 256
                          when two CTAs fit an SM, else 512)                             */
    int seg_flags;     /* BFS_SEG_SINGLE_BUFFER: one input buffer per CTA (the next
                          tile loads after the current one is merged; half the shared
                          memory, so two CTAs fit an SM)                                 */
} bfs_fdmt_desc;
enum { BFS_SEG_SINGLE_BUFFER = 1 };

typedef struct bfs_fdmt_plan bfs_fdmt_plan;

typedef struct bfs_fdmt_info {
    int niter;              /* number of merge levels (ceil(log2 nchan))      */
    int rows_level0;        /* rows of the level-0 plane                      */
    int fuse_depth;         /* fused levels actually used                     */
    int64_t rows_total;     /* sum of rows over levels 0..niter               */
    size_t workspace_bytes; /* device scratch the plan owns                   */
    double alg_bytes;       /* level-by-level algorithmic bytes of one call   */
    int out_rows;           /* output rows (max_dt; Pravir: the grid length)  */
    int hbm_passes;         /* merge passes after the head (each reads and writes HBM) */
    int seg_levels;         /* most merge levels fused into one of those passes */
    double sched_bytes;     /* DRAM bytes this schedule cannot avoid: the input read,
                               every plane that reaches HBM written and read once,
                               the output written                              */
} bfs_fdmt_info;

bfs_status bfs_fdmt_plan_create(const bfs_fdmt_desc* desc, bfs_fdmt_plan** plan);
/* The autotuner alone (no reference counterpart): times fusion depths
 * {0,2,3,4,5} x head tiles {256,512} x merge segments of 1..4 levels on this shape with zero input (the
 * kernels' cost does not depend on the values) and returns the fastest;
 * results are cached per (nchan, max_dt, band, ncols rounded up to 2^k). */
bfs_status bfs_fdmt_autotune(const bfs_fdmt_desc* desc, int* depth, int* head_tile, float* ms);
/* The same measurement over fusion depth, head tile and fused merge-segment
 * length (1..4 levels per HBM pass, FP32): *tuned = *desc with fuse_depth,
 * head_tile, seg_levels and seg_rows set to the fastest (cached per shape). */
bfs_status bfs_fdmt_autotune_desc(const bfs_fdmt_desc* desc, bfs_fdmt_desc* tuned, float* ms);
/* Same plan without device resources (introspection only; execute fails). */
bfs_status bfs_fdmt_plan_create_host(const bfs_fdmt_desc* desc, bfs_fdmt_plan** plan);
bfs_status bfs_fdmt_plan_destroy(bfs_fdmt_plan* plan);
bfs_status bfs_fdmt_plan_info(const bfs_fdmt_plan* plan, bfs_fdmt_info* info);
/* rows_per_level[0..niter] (cap entries at most); returns BFS_ERR_ARG if cap too small */
bfs_status bfs_fdmt_plan_rows(const bfs_fdmt_plan* plan, int* rows_per_level, int cap);
/* Delays of the output rows (out_cap >= out_rows; the reference's
 * FDMT::get_dt_grid_final, L/FDMT_PRAVIR/fdmt_base.cpp:61-63) and of the
 * level-0 rows with the level-0 row cumsum over channels (nchan + 1).  Any
 * pointer may be null. */
bfs_status bfs_fdmt_plan_delays(const bfs_fdmt_plan* plan, int* out_dt, int out_cap, int* lvl0_cum,
                                int* lvl0_dt, int lvl0_cap);
/* Host copies of level `level`'s (>= 1) row tables: tail row, head row (-1 = copied row), head shift. */
bfs_status bfs_fdmt_plan_tables(const bfs_fdmt_plan* plan, int level, int* a_row, int* b_row,
                                int* shift, int cap);
/* Fused-head layout (no reference counterpart; introspection for tests and
 * tuning): params[0..8] = depth, channels per group, tile, threads per CTA,
 * shared rows A, shared rows B, shared bytes, groups, table rows.  groups
 * (optional) receives per group {halo, out_row0, rows[9], tab_off[9]}; tab
 * (optional) receives 4 ints per row {tail, head, shift, 0} local to a group. */
bfs_status bfs_fdmt_plan_head(const bfs_fdmt_plan* plan, int* params, int* groups, int group_cap,
                              int* tab, int tab_cap);
/* Merge passes after the fused head (no reference counterpart; introspection
 * for tests and tuning): *npasses receives their number; params (optional,
 * cap ints) 13 ints per pass {first input level l0, output level l1, output
 * rows per tile, samples per tile, 32-column chunks per shared row, shared
 * row pitch, shared rows of buffer X, of buffer Y, most entries of a tile,
 * largest threshold, tiles, entries, level-0 rows per channel of an input
 * segment (0: the pass reads a level plane)}.  A pass with 0 tiles is one
 * plain merge level; the others fuse levels l0+1..l1 in shared memory; an
 * input segment reads the filterbank's channels and forms level 0 itself. */
bfs_status bfs_fdmt_plan_passes(const bfs_fdmt_plan* plan, int* npasses, int* params, int cap);
/* One fused pass's tiles (8 ints each: first entry, input rows, then the
 * rows of levels l0+1.. up to 6 levels) and entries (4 ints each: input rows
 * {plane row, window lead, 0, offset in buffer X}; level rows {tail offset,
 * head offset minus the shift (both in the buffer of the level below), shift
 * + lead, offset in this level's buffer or the output plane row}).  Each
 * shared buffer holds its rows, a row of -0.0 and a guard row. */
bfs_status bfs_fdmt_plan_segment(const bfs_fdmt_plan* plan, int pass, int* tiles, int tiles_cap,
                                 int* ent, int ent_cap);
/* d_in: nchan*ncols floats (ignored when b_ones != 0: an all-ones image is used,
 * the reference's normalisation mode), d_out: max_dt*ncols floats. */
bfs_status bfs_fdmt_execute(bfs_fdmt_plan* plan, const float* d_in, float* d_out, int b_ones,
                            void* stream);
/* Bytes of device scratch one call needs (the two ping-pong planes). */
bfs_status bfs_fdmt_workspace_size(const bfs_fdmt_plan* plan, size_t* bytes);
/* As bfs_fdmt_execute, with caller-provided scratch (>= workspace_size bytes,
 * 256-byte aligned).  Several plans may share one workspace on one stream. */
bfs_status bfs_fdmt_execute_ws(bfs_fdmt_plan* plan, const float* d_in, float* d_out, int b_ones,
                               void* d_workspace, size_t workspace_bytes, void* stream);

/* FDMT of a plane whose row c is all 1 where d_mask[c * mask_pitch] != 0 and
 * all 0 elsewhere (a row mask such as calc_fdmt_inputs' zapping mask): the
 * output is exactly what bfs_fdmt_execute gives on that plane (b_ones mode
 * is the all-1 case and uses the same path) — every value is an integer
 * count of channels, formed from the plan's per-channel delays in one pass
 * over the output instead of the level-by-level transform.  FP32 plans; the
 * first call uploads the delay table (allocates, synchronous). */
bfs_status bfs_fdmt_execute_row_mask(bfs_fdmt_plan* plan, const float* d_mask, int mask_pitch,
                                     float* d_out, void* stream);

/* Allocation-free FDMT.  No counterpart in the reference: it exists for
 * callers that cannot allocate device memory where they run the transform
 * (a real-time receiver whose GPU memory is all reserved at start-up, a
 * framework that owns the device allocator, a C caller with no CUDA
 * allocation code of its own).  `plan` may be host-only
 * (bfs_fdmt_plan_create_host).  The call allocates nothing: the row tables
 * and both ping-pong planes live in one 256 MiB static device array built
 * into the library (held by every GPU that loads it, until exit); a problem
 * needing more returns BFS_ERR_ARG.  The first call on each device looks the
 * array's device address up (cudaGetSymbolAddress) and keeps it for the life
 * of the process, so do not call cudaDeviceReset after using this entry
 * point.  Calls share the
 * array: calls that overlap on the GPU race.  Same output as
 * bfs_fdmt_execute (with b_ones != 0 too, d_in may then be NULL). */
bfs_status bfs_fdmt_execute_noalloc(const bfs_fdmt_plan* plan, const float* d_in, float* d_out,
                                    int b_ones, void* stream);
/* Scratch bytes bfs_fdmt_execute_noalloc needs for `plan`, and the static capacity. */
bfs_status bfs_fdmt_noalloc_scratch_bytes(const bfs_fdmt_plan* plan, size_t* need,
                                          size_t* capacity);

/* Adjoint (transpose) of the FDMT: d_grad_in (nchan x ncols) = F^T d_grad_out
 * (max_dt x ncols), with F the plan's linear transform (b_ones = 0).  No
 * reference counterpart (the reference has no gradients).  Each level's
 * adjoint is a gather over inverse row tables in a fixed order, so the FP32
 * result is deterministic; it needs no forward planes (every level is
 * linear).  Computed in FP32 whatever the plan's precision.  The first
 * adjoint call on a plan uploads its inverse tables (allocates, synchronous);
 * bfs_fdmt_adjoint also allocates the plan's adjoint planes then, so make
 * that first call outside any stream capture. */
bfs_status bfs_fdmt_adjoint(bfs_fdmt_plan* plan, const float* d_grad_out, float* d_grad_in,
                            void* stream);
bfs_status bfs_fdmt_adjoint_workspace_size(const bfs_fdmt_plan* plan, size_t* bytes);
bfs_status bfs_fdmt_adjoint_ws(bfs_fdmt_plan* plan, const float* d_grad_out, float* d_grad_in,
                               void* d_workspace, size_t workspace_bytes, void* stream);

/* ------------------------------------------------------------------------
 * Statistical preprocessing of the FDMT input.
 * Replaces statistical_preprocessing::calc_fdmt_inputs
 * (L/CDMT/Statistical_preprocessing.cuh:9-10, .cu:15-88): per-row mean and
 * variance, global mean/std, rows whose variance is > 4 sigma from the mean
 * variance are zeroed (mask 0), the rest become (x - mean)/std (mask 1).
 * d_buff: 4 + 2*nrows floats, same layout as the reference:
 * [row mean][row variance][mean][std][variance mean][variance std].
 * ---------------------------------------------------------------------- */
bfs_status bfs_preproc_calc_fdmt_inputs(float* d_inout, int nrows, int ncols, float* d_buff,
                                        float* d_norm_input, void* stream);
/* Replaces fdmt_normalization (L/CDMT/Chunk_gpu.cu:842-852):
 * d_out[i] = d_fdmt[i] / sqrtf(d_norm[i] + 1e-8).  d_out may alias d_fdmt. */
bfs_status bfs_fdmt_normalize(const float* d_fdmt, const float* d_norm, int64_t n, float* d_out,
                              void* stream);

/* ------------------------------------------------------------------------
 * Per-delay-row normalisation of a DM-time plane: out = (x - mean_r)/std_r
 * with FP64 row statistics (population std).  d_stats (optional, 2*rows
 * floats) receives [mean_r][std_r].  No reference counterpart: the
 * reference normalises the FDMT input instead (calc_fdmt_inputs above).
 * ---------------------------------------------------------------------- */
bfs_status bfs_norm_rows(const float* d_in, float* d_out, int rows, int cols, float* d_stats,
                         void* stream);
/* Only the statistics (2*rows floats: mean then std). */
bfs_status bfs_row_stats(const float* d_in, int rows, int cols, float* d_stats, void* stream);

/* ------------------------------------------------------------------------
 * Boxcar detection + candidate compaction.
 * widths_mode BFS_WIDTHS_POW2, param Q: widths 1,2,4..2^Q, mwidth = log2 w —
 *   replaces clusterization::gather_candidates_in_dynamicalArray
 *   (L/Clusterization/Clusterization.cu:56-89, :420-455).
 * widths_mode BFS_WIDTHS_ALL, param W: widths 1..W, mwidth = w —
 *   replaces gather_candidates_in_heap_with_plan (Clusterization.cu:169-202,
 *   :592-671).
 * The window sum is accumulated sequentially from the start sample (the
 * reference's order); only complete windows are tested; S/N = sum/sqrtf(w)
 * with an IEEE divide, as the reference's fdividef without --use_fast_math
 * (snr_fast != 0: the approximate __fdividef, <= 2 ulp, not bit-compatible).
 * A candidate is emitted when S/N > thr; thr is read from d_thr (device) when
 * non-NULL, else from `thr`.  d_stats (optional, from bfs_row_stats) makes the
 * kernel normalise each sample as (x - mean_r)/std_r before summing.
 * Candidates are returned in canonical row-major order (mdt, mt, width) —
 * the reference's heap order; the reference's atomic (dynamic) order is not
 * reproducible.  *h_count receives the total number found; if it exceeds
 * capacity only `capacity` are written and BFS_ERR_OVERFLOW is returned.
 * Synchronises `stream` (the count is returned to the host).
 * ---------------------------------------------------------------------- */
enum { BFS_WIDTHS_POW2 = 0, BFS_WIDTHS_ALL = 1 };
bfs_status bfs_boxcar_gather(const float* d_plane, int rows, int cols, const float* d_stats,
                             float thr, const float* d_thr, int widths_mode, int param,
                             int snr_fast, bfs_cand* d_out, uint32_t capacity,
                             uint32_t* h_count, void* stream);

/* Boxcar S/N at given cells and its gradient (no reference counterpart).
 * d_cells: n x {row, start, width} (device ints); d_stats: 2*rows floats
 * {means, stds} as bfs_row_stats writes.  S = sum_{j<width} (y - m)/s over
 * samples start..start+width-1, / sqrt(width), evaluated as the boxcar
 * kernels evaluate it (a cell outside the plane gives NaN).  The adjoint
 * writes the whole d_gplane (rows x cols) with d(sum_k gsnr_k S_k)/dy,
 * including the dependence of each row's mean and std on the row (at most
 * 512 cells per row; synchronises `stream`). */
bfs_status bfs_boxcar_snr_cells(const float* d_plane, int rows, int cols, const float* d_stats,
                                const int* d_cells, int n, float* d_snr, void* stream);
bfs_status bfs_boxcar_snr_cells_adjoint(const float* d_plane, int rows, int cols,
                                        const float* d_stats, const int* d_cells, int n,
                                        const float* d_snr, const float* d_gsnr, float* d_gplane,
                                        void* stream);

/* ------------------------------------------------------------------------
 * Clustering + delegates.
 * Replaces clusterization::complete_clusterization (Clusterization.cu:92-166):
 * three passes over (mt, mdt, mwidth) — sort inside each group, split where
 * consecutive keys differ by more than metrics[k] — then per-group argmax of
 * msnr (select_delegates_kernel, L/Clusterization/select_delegates.cu:63-125,
 * 64 lanes) and delegates sorted by mt (Clusterization.cu:147-149).  Ties are
 * broken by candidate index (canonical order).
 * Outputs (device, capacity n): d_perm (n) = members in group order,
 * d_offsets (n+1) = group starts, d_delegates (n) = delegate candidate index
 * per group sorted by (mt, group).  *h_ngroups receives the group count.
 * Synchronises `stream`.
 * ---------------------------------------------------------------------- */
bfs_status bfs_cluster(const bfs_cand* d_cands, uint32_t n, const int* metrics /* host, 3 */,
                       int* d_perm, int* d_offsets, int* d_delegates, uint32_t* h_ngroups,
                       void* stream);
/* bfs_cluster with initial groups (no reference counterpart; used by the
 * batched runner to cluster many beams at once): candidate i starts in group
 * d_group0[i] (0..ngroups0-1, non-decreasing in the candidate order), so no
 * group ever spans two initial groups.  d_group0 = NULL is bfs_cluster. */
bfs_status bfs_cluster_grouped(const bfs_cand* d_cands, uint32_t n, const int* d_group0,
                               uint32_t ngroups0, const int* metrics, int* d_perm, int* d_offsets,
                               int* d_delegates, uint32_t* h_ngroups, void* stream);
/* The reference's per-group argmax on its own (select_delegates_kernel).
 * The device arrays are read as bfs_cluster writes them and are not checked:
 * d_offsets holds ngroups + 1 non-decreasing entries from 0 to n, and every
 * d_perm entry is an index into d_cands (0..n-1).  Other contents read
 * outside the arrays. */
bfs_status bfs_select_delegates(const bfs_cand* d_cands, const int* d_perm, uint32_t n,
                                const int* d_offsets, uint32_t ngroups, int* d_delegates,
                                void* stream);

/* ------------------------------------------------------------------------
 * Batched multi-beam search (no single reference counterpart: it batches the
 * reference's per-chunk FDMT + clusterization_main sequence over many beams).
 * Every beam's FDMT (autotuned plans sharing one workspace), row statistics
 * and boxcar are captured once into a CUDA graph and replayed; the candidates
 * of all beams are sorted and clustered in one pass (beams are the initial
 * groups, so no cluster spans two beams).  Results per beam: delegates in
 * (mt, group) order with their group sizes.
 * ---------------------------------------------------------------------- */
typedef struct bfs_batch_desc {
    int nbeams;
    const bfs_fdmt_desc* beams;  /* per-beam FDMT descriptions (fuse_depth as usual) */
    int widths_mode;             /* BFS_WIDTHS_POW2 / BFS_WIDTHS_ALL                  */
    int param;                   /* Q or W                                           */
    float thr;                   /* S/N threshold on the row-normalised planes       */
    int metrics[3];              /* clustering metrics (mt, mdt, mwidth)             */
    uint32_t capacity;           /* candidates over all beams (0 = 2^26)             */
    int use_graph;               /* capture stage 1 in a CUDA graph                  */
    int reserved[8];
} bfs_batch_desc;

typedef struct bfs_batch bfs_batch;

bfs_status bfs_batch_create(const bfs_batch_desc* desc, bfs_batch** batch);
bfs_status bfs_batch_destroy(bfs_batch* batch);
/* d_inputs: host array of nbeams device pointers (nchan x ncols each).  The
 * first run is eager; later runs replay the captured graph while the input
 * pointers are unchanged (a new set is captured again).  Synchronises. */
bfs_status bfs_batch_run(bfs_batch* batch, const float* const* d_inputs, void* stream);
/* The same with host inputs: h_inputs[i] (pinned host memory, nchan x ncols)
 * is copied into d_inputs[i] (device) on an internal copy stream while the
 * beams before it are searched, so the copies overlap the compute; copies
 * and compute are captured in one CUDA graph after the first run.
 * Synchronises `stream`. */
bfs_status bfs_batch_run_host(bfs_batch* batch, const float* const* h_inputs,
                              float* const* d_inputs, void* stream);
/* The asynchronous form (no reference counterpart): bfs_batch_submit
 * enqueues one run's FDMT + statistics + boxcar of every beam on an internal
 * stream (after the work already on `stream`, which makes the inputs ready)
 * and returns; bfs_batch_collect waits for the oldest submitted run and does
 * its sort, clustering and delegates on `stream`, leaving its results for
 * bfs_batch_counts / bfs_batch_beam_results as bfs_batch_run does.  At most
 * two runs are in flight (two candidate buffers), so submit(i + 1) before
 * collect(i) overlaps run i's clustering with run i + 1's FDMT.  The inputs
 * of a run must stay unchanged until it is collected.  bfs_batch_run and
 * bfs_batch_run_host refuse to start while runs are in flight. */
bfs_status bfs_batch_submit(bfs_batch* batch, const float* const* d_inputs, void* stream);
bfs_status bfs_batch_collect(bfs_batch* batch, void* stream);
bfs_status bfs_batch_counts(const bfs_batch* batch, uint32_t* n_cands, uint32_t* n_groups);
/* Host copies of one beam's delegates (cap entries) and group sizes. */
bfs_status bfs_batch_beam_results(const bfs_batch* batch, int beam, bfs_cand* delegates,
                                  int* group_sizes, int cap, int* n_delegates,
                                  uint32_t* n_candidates);

/* Square fragment of a DM-time plane around (target_row, target_col) for
 * vetting (CChunkB::cutQuadraticFragment, L/CDMT/ChunkB.cpp:255-275, and
 * CFragment, L/Fragment.h:3-28): dim = min(rows, cols); with rows < cols the
 * rows x rows block from column (target_col / rows) * rows, else the
 * cols x cols block at the top; read at the reference's flat row-major
 * positions, 0 past the end of the plane.  d_out (device, dim*dim) may be
 * null to get the geometry only. */
bfs_status bfs_cut_fragment(const float* d_plane, int rows, int cols, int target_row, int target_col,
                            float* d_out, int* row_begin, int* col_begin, int* dim, void* stream);

/* ------------------------------------------------------------------------
 * GUPPI RAW input (replaces CSession_guppi's file handling,
 * L/CDMT/Session_guppi.cpp:31-85,111-283,336-369 and
 * L/TelescopeHeader.cpp:88-124,175-347).  Header keys as the reference reads
 * them (DIRECTIO, NBITS, CHAN_BW, OBSFREQ, OBSNCHAN, OBSBW, BLOCSIZE,
 * TELESCOP, NPOL, TBIN; data after the third "END", 512-byte aligned with
 * DIRECTIO).  8-bit samples.  Chunks are [nchan][len_chunk][npol] int8 in
 * ascending frequency (a negative CHAN_BW reverses the stored order); chunk j
 * of a block starts at sample j*(len_chunk - 2*noverlap), the last ends at
 * the block's last sample (the reference's session loop; its rewind before
 * the last chunk of a block is not reproduced).
 * ---------------------------------------------------------------------- */
enum { BFS_GUPPI_GBT = 0, BFS_GUPPI_PARKES = 1 };
typedef struct bfs_guppi_header {
    int nbits;
    float chan_bw;        /* |CHAN_BW| (MHz)                                     */
    int npol;             /* bytes per sample per channel at 8 bits (NPOL)       */
    int directio;
    float obsfreq;        /* |OBSFREQ| (MHz), band centre                        */
    int nchan;            /* OBSNCHAN                                            */
    float obsbw;          /* |OBSBW| (MHz)                                       */
    int64_t blocsize;     /* data bytes of the block                             */
    int telescope;        /* BFS_GUPPI_GBT / BFS_GUPPI_PARKES                    */
    float tbin;           /* sample time (s)                                     */
    int straight_order;   /* 1: ascending frequency in the file (CHAN_BW >= 0)   */
    int64_t data_offset;  /* byte offset of the block's data                     */
    int64_t nsamp;        /* samples per channel in the block                    */
    float fmin, fmax;     /* obsfreq -/+ obsbw / 2                               */
    int reserved[4];
} bfs_guppi_header;
typedef struct bfs_guppi_file bfs_guppi_file;
typedef struct bfs_guppi_reader bfs_guppi_reader;

/* Parses one header held in text[0..len) (data_offset relative to text). */
bfs_status bfs_guppi_parse_header(const char* text, size_t len, bfs_guppi_header* out);
/* Opens a file and indexes its blocks (CSession_guppi::calcQuantBlocks). */
bfs_status bfs_guppi_open(const char* path, bfs_guppi_file** out);
bfs_status bfs_guppi_close(bfs_guppi_file* file);
bfs_status bfs_guppi_blocks(const bfs_guppi_file* file, int* nblocks);
bfs_status bfs_guppi_block_header(const bfs_guppi_file* file, int block, bfs_guppi_header* out);
bfs_status bfs_guppi_chunk_count(const bfs_guppi_file* file, int block, int64_t len_chunk,
                                 int64_t noverlap, int64_t* nchunks);
/* One chunk into host memory dst (CSession_guppi::download_chunk). */
bfs_status bfs_guppi_read_chunk(const bfs_guppi_file* file, int block, int64_t chunk, int64_t len_chunk,
                                int64_t noverlap, int8_t* dst, size_t dst_bytes);
/* Streaming reader (no reference counterpart): a background thread reads
 * every chunk of every block in order into `nbuffers` host buffers (pinned
 * when `pinned`); _next hands out the next one and, given d_dst (device,
 * chunk-sized), copies it there asynchronously on `stream`, so file reads,
 * copies and the caller's kernels overlap.  *block = -1 at the end.  The
 * host buffer (h_src) stays valid until the next call. */
bfs_status bfs_guppi_reader_create(const bfs_guppi_file* file, int64_t len_chunk, int64_t noverlap,
                                   int nbuffers, int pinned, bfs_guppi_reader** out);
bfs_status bfs_guppi_reader_next(bfs_guppi_reader* reader, void* d_dst, void* stream,
                                 const int8_t** h_src, int* block, int64_t* chunk);
bfs_status bfs_guppi_reader_destroy(bfs_guppi_reader* reader);

/* Chunk geometry of a GUPPI session, as CSessionB::launch derives it from the
 * first block's header, the pulse length t_p (s), the DM range, nbin and nfft
 * (L/CDMT/SessionB.cpp:144-160,184-206; get_optimal_overlap :384-392;
 * get_coherent_dms :395-401), in the reference's float/double arithmetic:
 *   len_sft   = ceil(t_p / TBIN)
 *   optimal   = round(delay(d_max, fmin, fmin + OBSBW/(OBSNCHAN len_sft)) / TBIN)
 *   noverlap  = 2^round(log2(optimal / 2))  (0 when optimal / 2 is 0)
 *   len_chunk = (nbin - 2 noverlap) nfft
 *   ncoherent = ceil(delay(d_max, fmin, fmax) TBIN / t_p^2)
 * with delay(dm, a, b) = 4.148808e3 dm (1/a^2 - 1/b^2) s, a and b in MHz.
 * d_min / d_max are returned as the chunk receives them (float).  Errors
 * where the reference would divide by zero or run a chunk of negative length
 * (d_max <= 0, 2 noverlap >= nbin). */
typedef struct bfs_guppi_session {
    int len_sft;          /* fine channels per coarse channel                    */
    int noverlap;         /* overlap-save samples on each side of a segment      */
    int64_t len_chunk;    /* samples per channel in one chunk                    */
    int ncoherent;        /* coherent-DM count handed to the chunk               */
    int optimal_overlap;  /* get_optimal_overlap(len_sft), samples               */
    float fmin, fmax;     /* band edges handed to the chunk (MHz)                */
    float tsamp;          /* TBIN (s)                                            */
    float d_min, d_max;   /* DM range as the chunk receives it                   */
    int reserved[4];
} bfs_guppi_session;
bfs_status bfs_guppi_session_plan(const bfs_guppi_header* header, float pulse_length, double d_min,
                                  double d_max, int nbin, int nfft, bfs_guppi_session* out);

/* ------------------------------------------------------------------------
 * Coherent-dedispersion chunk stage.
 * Replaces CSession_guppi_gpu::unpack_chunk (L/CDMT/Session_guppi_gpu.cu:53-60,
 * 117-141) and CChunk_gpu / CChunk_fly_gpu::process (L/CDMT/Chunk_gpu.cu:134-460,
 * L/CDMT/Chunk_fly_gpu.cu:94-163) with the CChunkB geometry
 * (L/CDMT/ChunkB.h:77-98): mbin = nbin/len_sft, noverlap_per_channel =
 * noverlap/len_sft, mbin_adjusted = mbin - 2*noverlap_per_channel,
 * msamp = nfft*mbin_adjusted, rows = nchan*len_sft.
 * Buffers: raw chunk int8 [nchan][len_chunk][npol] with len_chunk =
 * (nbin - 2*noverlap)*nfft; spectra/voltages complex64 (float2)
 * [npol/2][nfft][nchan][nbin]; planes float32 [rows][msamp], row 0 = highest
 * frequency (the reference's reversed order).
 * ---------------------------------------------------------------------- */
typedef struct bfs_chunk_desc {
    float fmin;        /* MHz, band edges (CChunkB m_Fmin / m_Fmax)            */
    float fmax;
    int npol;          /* 2 = one complex polarisation, 4 = two                */
    int nchan;         /* coarse channels                                      */
    int len_sft;       /* fine channels per coarse channel                     */
    int nbin;          /* forward FFT length                                   */
    int nfft;          /* FFT segments per chunk                               */
    int noverlap;      /* overlap-save samples on each side of a segment       */
    float tsamp;       /* coarse-channel sample time, seconds                  */
    int max_dt;        /* FDMT output rows (0 = len_sft, the reference's value) */
    int reserved[6];
} bfs_chunk_desc;

typedef struct bfs_chunk bfs_chunk;

bfs_status bfs_chunk_create(const bfs_chunk_desc* desc, bfs_chunk** chunk);
bfs_status bfs_chunk_destroy(bfs_chunk* chunk);
/* info[0..7] = mbin, noverlap_per_channel, mbin_adjusted, msamp, rows,
 * len_chunk, complex values per buffer, max_dt */
bfs_status bfs_chunk_info(const bfs_chunk* chunk, int64_t* info, int cap);
/* Coherent-DM grid of CChunkB::CChunkB (L/CDMT/ChunkB.cpp:171-176); returns the count. */
int bfs_chunk_coherent_dms(double d_min, double d_max, int ncoherent, double* dms, int cap);
/* GUPPI unpack with overlap-save zero padding (unpack_chunk_guppi_gpu). */
bfs_status bfs_chunk_unpack(bfs_chunk* chunk, const int8_t* d_raw, void* d_cplx, void* stream);
/* In-place forward FFT of every segment (Chunk_gpu.cu:267). */
bfs_status bfs_chunk_forward_fft(bfs_chunk* chunk, void* d_cplx, void* stream);
/* Coherently dedispersed voltages for one DM: chirp (FP64 phase) + inverse
 * FFTs of length mbin (Chunk_fly_gpu.cu:94-163, Chunk_gpu.cu:284-288).
 * d_spec is not modified.  For mbin = 32768 (nbin a power of two, d_spec
 * 16-byte aligned, d_volt not overlapping d_spec) the library's own two-pass
 * transform with the chirp applied on load; it agrees with chirp + cuFFT to
 * FP32 rounding.  Other cases: chirp + cuFFT. */
bfs_status bfs_chunk_voltages(bfs_chunk* chunk, const void* d_spec, double dm, void* d_volt,
                              void* stream);
/* Power detection + roll + unpadding + frequency reversal + dedispersion shift
 * (Chunk_gpu.cu:296-321) into a rows x msamp plane.  Synchronises `stream`. */
bfs_status bfs_chunk_detect(bfs_chunk* chunk, const void* d_volt, double dm, float* d_plane,
                            void* stream);
/* bfs_chunk_voltages followed by bfs_chunk_detect without storing the
 * voltages where the own sub-band transform applies (its second pass writes
 * the detected plane): the same plane, bit for bit, as detecting the
 * voltages bfs_chunk_voltages returns.  Synchronises `stream`. */
bfs_status bfs_chunk_detect_spectrum(bfs_chunk* chunk, const void* d_spec, double dm, float* d_plane,
                                     void* stream);
/* CChunkB::process (L/CDMT/ChunkB.h:73-74): forward FFT of d_cplx (in place,
 * overwritten like the reference's), then per DM voltages, detection,
 * statistical preprocessing, FDMT of mask and data and fdmt_normalization into
 * d_out[i] (max_dt x msamp each). */
bfs_status bfs_chunk_process(bfs_chunk* chunk, void* d_cplx, const double* dms, int ndm,
                             float* d_out, void* stream);
/* unpack_chunk_guppi_gpu (Session_guppi_gpu.cu:117-141) followed by the
 * forward FFT of CChunk_gpu::process (Chunk_gpu.cu:267), as one step: d_spec
 * (complex values per buffer, bfs_chunk_info[6]) receives the spectra of every
 * segment.  For nbin = 2^20 a four-step transform whose first pass reads the
 * int8 samples directly (no complex copy of the chunk); it agrees with
 * bfs_chunk_unpack + bfs_chunk_forward_fft to FP32 rounding.  Other sizes (or a
 * d_raw not aligned to npol bytes, a d_spec not aligned to 8) run those two.
 * Uses the chunk's voltage buffer as scratch.  The first call on a device
 * builds the transform's twiddle tables (allocates, synchronous; kept until
 * exit): make it before any stream capture. */
bfs_status bfs_chunk_unpack_fft(bfs_chunk* chunk, const int8_t* d_raw, void* d_spec, void* stream);
/* The per-DM part of CChunkB::process (Chunk_gpu.cu:284-359) on spectra from
 * bfs_chunk_unpack_fft or bfs_chunk_forward_fft: d_spec is not modified. */
bfs_status bfs_chunk_process_spectrum(bfs_chunk* chunk, const void* d_spec, const double* dms, int ndm,
                                      float* d_out, void* stream);
/* CSession_guppi_gpu::unpack_chunk + CChunkB::process from the raw chunk:
 * bfs_chunk_unpack_fft into d_spec, then per DM what bfs_chunk_process does
 * after its forward FFT. */
bfs_status bfs_chunk_process_raw(bfs_chunk* chunk, const int8_t* d_raw, void* d_spec, const double* dms,
                                 int ndm, float* d_out, void* stream);

/* ---- self-tests (no reference counterpart) ---- */

/* Compares the level-0 kernels' division by the constant d (a multiply and a
 * fused multiply-add for d = 2..8, __fdiv_rn otherwise) with __fdiv_rn(x, d)
 * for all 2^32 float bit patterns x on the current device; *mismatches = how
 * many differ (0 means the FDMT's level 0 is bit-exact for that divisor),
 * *first_bad (may be NULL) = the lowest differing bit pattern.  Synchronises
 * `stream`. */
bfs_status bfs_selftest_divide(int d, uint64_t* mismatches, uint32_t* first_bad, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* BFS_H */
