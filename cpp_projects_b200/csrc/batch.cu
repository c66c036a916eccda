// Batched multi-beam search: many beams of uneven channel counts and lengths
// through FDMT -> per-row statistics -> normalise + boxcar + compaction ->
// clustering, with the per-beam kernel sequence of every beam captured in ONE
// CUDA graph and the candidate handling done once for the whole batch.
//
// The reference runs one chunk at a time with host round trips between
// stages (CChunk_gpu::process, L/CDMT/Chunk_gpu.cu:254-460; clusterization_main,
// L/Clusterization/Clusterization.cu:17-54).  Here:
//   stage 1 (graph)  for each beam: fused/plain FDMT into a shared DM-time
//                    plane, row statistics, and the boxcar appending to one
//                    device-wide candidate array with a shared atomic counter
//                    — no host sync.  Width sets with an ordered boxcar write
//                    each tile's candidates as one block in canonical order
//                    and record (first, count) per (beam, row, tile); others
//                    tag every candidate with its beam;
//   stage 2          one read of the counter, the canonical order over all
//                    beams (beam, row, sample, width) — a scan of the record
//                    counts and one move of every block, or a radix sort of
//                    the tagged candidates —, one 3-pass clustering whose
//                    initial groups are the beams, one delegate sort by
//                    (beam, mt, group), one copy of the delegates to the host.
// Plans are autotuned per shape and share one workspace; the DM-time plane
// and statistics buffers are shared (the graph serialises the beams on one
// stream), so device memory is set by the largest beam plus the candidates.
#include <cub/device/device_radix_sort.cuh>

#include <memory>
#include <vector>

#include "internal.h"

namespace bfs {
bfs_status launch_row_stats(const float* d_in, int rows, int cols, float* d_stats, int mode,
                            cudaStream_t s);
bfs_status launch_boxcar(const float* d_plane, int rows, int cols, const float* d_stats,
                         float thr, const float* d_thr, int mode, int param, int snr_fast,
                         bfs_cand* d_out, unsigned capacity, unsigned* d_count, cudaStream_t s,
                         int tag, int* d_tags);
bfs_status sort_tagged_candidates(const bfs_cand* d_c, const int* d_tags, unsigned n, int max_rows,
                                  int max_cols, int max_tag, int mode, int param, bfs_cand* d_dst,
                                  int* d_tdst, cudaStream_t s);
bool boxcar_ordered_supported(int mode, int param);
long long boxcar_ordered_records(int rows, int cols);
bfs_status launch_boxcar_ordered(const float* d_plane, int rows, int cols, const float* d_stats, float thr,
                                 const float* d_thr, int mode, int param, int snr_fast, bfs_cand* d_out,
                                 unsigned capacity, unsigned* d_count, unsigned* rec_first, unsigned* rec_count,
                                 cudaStream_t s);
bfs_status compact_ordered(const bfs_cand* src, const unsigned* rec_first, const unsigned* rec_count,
                           long long nrec, const long long* beam_rec, int nb, bfs_cand* dst, int* tags,
                           cudaStream_t s);
}  // namespace bfs

struct bfs_batch {
    std::vector<bfs_fdmt_desc> beams;
    std::vector<bfs_fdmt_plan*> plans;
    int widths_mode = 0, param = 5;
    float thr = 7.0f;
    int metrics[3] = {16, 8, 1 << 30};
    unsigned capacity = 0;
    bool use_graph = true;
    int max_rows = 0, max_cols = 0;
    void* ws = nullptr;
    size_t ws_bytes = 0;
    float* plane = nullptr;
    float* stats = nullptr;
    bfs_cand* cands = nullptr;     // boxcar output (arrival order)
    int* tags = nullptr;           // (tagged-sort path) each candidate's beam
    // ordered path: per-tile records of the boxcar's canonical blocks
    bool ordered = false;
    long long nrec = 0;
    std::vector<long long> rec0;   // first record of each beam (+ the total)
    unsigned* rec = nullptr;       // first[nrec], count[nrec]
    long long* d_beam_rec = nullptr;
    bfs_cand* sorted = nullptr;    // canonical order
    int* sorted_tags = nullptr;
    unsigned* d_count = nullptr;
    int *perm = nullptr, *offsets = nullptr, *delegates = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<const float*> graph_inputs;
    int runs = 0;
    // host-input form: copies + compute captured together (bfs_batch_run_host)
    cudaGraph_t hgraph = nullptr;
    cudaGraphExec_t hexec = nullptr;
    std::vector<const void*> hgraph_ptrs;   // host then device pointers it was captured for
    std::vector<cudaEvent_t> events;
    // the asynchronous form (bfs_batch_submit / bfs_batch_collect): two sets
    // of stage-1 buffers; the fields above hold set `active`, these the other
    bfs_cand* cands_alt = nullptr;
    int* tags_alt = nullptr;
    unsigned* rec_alt = nullptr;
    unsigned* d_count_alt = nullptr;
    cudaGraph_t graph_alt = nullptr;
    cudaGraphExec_t exec_alt = nullptr;
    std::vector<const float*> graph_inputs_alt;
    int active = 0;
    cudaStream_t s1 = nullptr;               // stage-1 stream of submitted runs
    cudaEvent_t ev_in = nullptr, ev_done[2] = {nullptr, nullptr};
    int queue[2] = {0, 0}, qhead = 0, inflight = 0, next_set = 0;
    // stage 1 in kLanes lanes (branches of the graph): lane l > 0 has its own
    // plane, statistics and FDMT workspace (lane 0 uses the ones above);
    // beam i runs in lane lane_of[i]
    static constexpr int kLanes = 2;
    float* lane_plane[kLanes] = {};
    float* lane_stats[kLanes] = {};
    void* lane_ws[kLanes] = {};
    std::vector<int> lane_of;
    cudaStream_t lane_s[kLanes] = {};
    cudaEvent_t ev_fork = nullptr, ev_join[kLanes] = {};
    // results of the last run
    unsigned n_cands = 0, n_groups = 0;
    std::vector<bfs_cand> h_delegates;
    std::vector<int> h_delegate_beam, h_delegate_size, h_beam_first, h_beam_count, h_beam_cands;
    ~bfs_batch() {
        // work still queued on the batch's own streams (a submitted run that
        // was never collected) must finish before its buffers are freed
        if (s1) cudaStreamSynchronize(s1);
        for (cudaStream_t t : lane_s)
            if (t) cudaStreamSynchronize(t);
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (hexec) cudaGraphExecDestroy(hexec);
        if (hgraph) cudaGraphDestroy(hgraph);
        if (exec_alt) cudaGraphExecDestroy(exec_alt);
        if (graph_alt) cudaGraphDestroy(graph_alt);
        for (cudaEvent_t e : {ev_in, ev_done[0], ev_done[1]})
            if (e) cudaEventDestroy(e);
        if (s1) cudaStreamDestroy(s1);
        if (ev_fork) cudaEventDestroy(ev_fork);
        for (int l = 0; l < kLanes; ++l) {
            if (ev_join[l]) cudaEventDestroy(ev_join[l]);
            if (lane_s[l]) cudaStreamDestroy(lane_s[l]);
            if (l > 0) {
                for (void* p : {static_cast<void*>(lane_plane[l]), static_cast<void*>(lane_stats[l]), lane_ws[l]})
                    if (p) cudaFree(p);
            }
        }
        for (void* p : {static_cast<void*>(cands_alt), static_cast<void*>(tags_alt), static_cast<void*>(rec_alt),
                        static_cast<void*>(d_count_alt)})
            if (p) cudaFree(p);
        for (cudaEvent_t e : events) cudaEventDestroy(e);
        for (auto* p : plans) bfs_fdmt_plan_destroy(p);
        for (void* p : {ws, static_cast<void*>(plane), static_cast<void*>(stats), static_cast<void*>(cands),
                        static_cast<void*>(tags), static_cast<void*>(rec), static_cast<void*>(d_beam_rec),
                        static_cast<void*>(sorted), static_cast<void*>(sorted_tags),
                        static_cast<void*>(d_count), static_cast<void*>(perm), static_cast<void*>(offsets),
                        static_cast<void*>(delegates)})
            if (p) cudaFree(p);
    }
};

namespace bfs {
namespace {

// Inverse of the group-order permutation: position of every candidate.
__global__ void k_inverse_perm(const int* __restrict__ perm, unsigned n, int* __restrict__ inv) {
    const unsigned p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < n) inv[perm[p]] = static_cast<int>(p);
}

// For delegate i (in the (mt, group) order bfs_cluster returns): its record,
// beam, group size, and the beam as the key of the final stable sort.
__global__ void k_delegate_info(const bfs_cand* __restrict__ c, const int* __restrict__ tags,
                                const int* __restrict__ dl, const int* __restrict__ inv,
                                const int* __restrict__ offsets, unsigned ng,
                                bfs_cand* __restrict__ rec, int* __restrict__ size,
                                unsigned* __restrict__ key, unsigned* __restrict__ val) {
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ng) return;
    const int di = dl[i];
    const int p = inv[di];
    int lo = 0, hi = static_cast<int>(ng) - 1;  // group = last offset <= p
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (offsets[mid] <= p) lo = mid; else hi = mid - 1;
    }
    rec[i] = c[di];
    size[i] = offsets[lo + 1] - offsets[lo];
    key[i] = static_cast<unsigned>(tags[di]);
    val[i] = i;
}

__global__ void k_permute_delegates(const bfs_cand* __restrict__ rec, const int* __restrict__ size,
                                    const unsigned* __restrict__ beam, const unsigned* __restrict__ order,
                                    unsigned ng, bfs_cand* __restrict__ rec_out, int* __restrict__ size_out,
                                    int* __restrict__ beam_out) {
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ng) return;
    rec_out[i] = rec[order[i]];
    size_out[i] = size[order[i]];
    beam_out[i] = static_cast<int>(beam[i]);
}

// Candidates per beam from the tag-sorted list (lower bounds).
__global__ void k_beam_bounds(const int* __restrict__ sorted_tags, unsigned n, int nb,
                              unsigned* __restrict__ first) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b > nb) return;
    unsigned lo = 0, hi = n;
    while (lo < hi) {
        const unsigned mid = (lo + hi) >> 1;
        if (sorted_tags[mid] < b) lo = mid + 1; else hi = mid;
    }
    first[b] = lo;
}

int bits_of(unsigned long long v) {
    int b = 0;
    while (b < 64 && (v >> b) != 0ull) ++b;
    return b;
}

}  // namespace
}  // namespace bfs

using namespace bfs;

extern "C" bfs_status bfs_batch_create(const bfs_batch_desc* desc, bfs_batch** out) {
    BFS_ARG(desc && out && desc->beams && desc->nbeams >= 1, "bad batch description");
    *out = nullptr;
    std::unique_ptr<bfs_batch> b(new bfs_batch);
    b->beams.assign(desc->beams, desc->beams + desc->nbeams);
    b->widths_mode = desc->widths_mode;
    b->param = desc->param;
    b->thr = desc->thr;
    for (int i = 0; i < 3; ++i) b->metrics[i] = desc->metrics[i];
    b->capacity = desc->capacity ? desc->capacity : (1u << 26);
    BFS_ARG(b->capacity < 0x7fffffffu, "capacity %u too large", b->capacity);
    b->use_graph = desc->use_graph != 0;
    size_t plane = 0;
    for (const bfs_fdmt_desc& d0 : b->beams) {
        bfs_fdmt_desc d = d0;
        d.flags |= BFS_FDMT_EXTERNAL_WS;
        bfs_fdmt_plan* p = nullptr;
        bfs_status st = bfs_fdmt_plan_create(&d, &p);
        if (st != BFS_OK) return st;
        b->plans.push_back(p);
        size_t need = 0;
        bfs_fdmt_workspace_size(p, &need);
        b->ws_bytes = std::max(b->ws_bytes, need);
        plane = std::max(plane, static_cast<size_t>(d.max_dt) * d.ncols);
        b->max_rows = std::max(b->max_rows, d.max_dt);
        b->max_cols = std::max(b->max_cols, d.ncols);
    }
    BFS_ARG(b->max_rows <= 65535, "max_dt above 65535");
    b->ordered = boxcar_ordered_supported(b->widths_mode, b->param);
    if (b->ordered) {
        for (const bfs_fdmt_desc& d : b->beams) {
            b->rec0.push_back(b->nrec);
            b->nrec += boxcar_ordered_records(d.max_dt, d.ncols);
        }
        b->rec0.push_back(b->nrec);
        BFS_ARG(b->nrec < (1ll << 31), "too many boxcar tiles in the batch (%lld)", b->nrec);
        BFS_CUDA(cudaMalloc(&b->rec, sizeof(unsigned) * 2 * b->nrec));
        BFS_CUDA(cudaMalloc(&b->d_beam_rec, sizeof(long long) * b->rec0.size()));
        BFS_CUDA(cudaMemcpy(b->d_beam_rec, b->rec0.data(), sizeof(long long) * b->rec0.size(),
                            cudaMemcpyHostToDevice));
    }
    BFS_CUDA(cudaMalloc(&b->ws, b->ws_bytes ? b->ws_bytes : 256));
    BFS_CUDA(cudaMalloc(&b->plane, plane * sizeof(float)));
    BFS_CUDA(cudaMalloc(&b->stats, 2 * static_cast<size_t>(b->max_rows) * sizeof(float)));
    // lanes: beams in order, each to the lane with the least work so far
    constexpr int L = bfs_batch::kLanes;
    b->lane_of.assign(b->beams.size(), 0);
    b->lane_plane[0] = b->plane;
    b->lane_stats[0] = b->stats;
    b->lane_ws[0] = b->ws;
    if (b->beams.size() >= 2) {
        double work[L] = {};
        for (size_t i = 0; i < b->beams.size(); ++i) {
            int l = 0;
            for (int k = 1; k < L; ++k)
                if (work[k] < work[l]) l = k;
            b->lane_of[i] = l;
            work[l] += static_cast<double>(b->beams[i].max_dt) * b->beams[i].ncols +
                       static_cast<double>(b->beams[i].nchan) * b->beams[i].ncols;
        }
        for (int l = 1; l < L; ++l) {
            BFS_CUDA(cudaMalloc(&b->lane_ws[l], b->ws_bytes ? b->ws_bytes : 256));
            BFS_CUDA(cudaMalloc(&b->lane_plane[l], plane * sizeof(float)));
            BFS_CUDA(cudaMalloc(&b->lane_stats[l], 2 * static_cast<size_t>(b->max_rows) * sizeof(float)));
        }
        for (auto& t : b->lane_s) BFS_CUDA(cudaStreamCreateWithFlags(&t, cudaStreamNonBlocking));
        BFS_CUDA(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming));
        for (auto& e : b->ev_join) BFS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    const size_t cap = b->capacity;
    BFS_CUDA(cudaMalloc(&b->cands, cap * sizeof(bfs_cand)));
    if (!b->ordered) BFS_CUDA(cudaMalloc(&b->tags, cap * sizeof(int)));
    BFS_CUDA(cudaMalloc(&b->sorted, cap * sizeof(bfs_cand)));
    BFS_CUDA(cudaMalloc(&b->sorted_tags, cap * sizeof(int)));
    BFS_CUDA(cudaMalloc(&b->d_count, sizeof(unsigned)));
    BFS_CUDA(cudaMalloc(&b->perm, cap * sizeof(int)));
    BFS_CUDA(cudaMalloc(&b->offsets, (cap + 1) * sizeof(int)));
    BFS_CUDA(cudaMalloc(&b->delegates, cap * sizeof(int)));
    *out = b.release();
    return BFS_OK;
}

extern "C" bfs_status bfs_batch_destroy(bfs_batch* b) {
    delete b;
    return BFS_OK;
}

// Boxcar of beam i over the shared plane: ordered blocks + records, or
// atomic appends tagged with the beam.
static bfs_status beam_boxcar(bfs_batch* b, int i, const float* plane, const float* stats, cudaStream_t s) {
    const bfs_fdmt_desc& d = b->beams[i];
    if (b->ordered)
        return launch_boxcar_ordered(plane, d.max_dt, d.ncols, stats, b->thr, nullptr, b->widths_mode,
                                     b->param, 0, b->cands, b->capacity, b->d_count, b->rec + b->rec0[i],
                                     b->rec + b->nrec + b->rec0[i], s);
    return launch_boxcar(plane, d.max_dt, d.ncols, stats, b->thr, nullptr, b->widths_mode, b->param, 0,
                         b->cands, b->capacity, b->d_count, s, i, b->tags);
}

// FDMT, row statistics and boxcar of beam i with one lane's plane,
// statistics and workspace.
static bfs_status beam_stage1(bfs_batch* b, int i, const float* d_in, float* plane, float* stats, void* ws,
                              cudaStream_t s) {
    const bfs_fdmt_desc& d = b->beams[i];
    bfs_status st = bfs_fdmt_execute_ws(b->plans[i], d_in, plane, 0, ws, b->ws_bytes, s);
    if (st != BFS_OK) return st;
    st = launch_row_stats(plane, d.max_dt, d.ncols, stats, 0, s);
    if (st != BFS_OK) return st;
    return beam_boxcar(b, i, plane, stats, s);
}

// Stage 1 for every beam, enqueued on s (captured or eager).
// With several lanes the beams fork from s into the lanes' streams (branches of
// the captured graph) and join back; the candidates of both lanes go to the
// one candidate array (their order is set by the records or the sort).
static bfs_status enqueue_stage1(bfs_batch* b, const float* const* d_inputs, cudaStream_t s) {
    BFS_CUDA(cudaMemsetAsync(b->d_count, 0, sizeof(unsigned), s));
    if (!b->lane_s[0]) {
        for (size_t i = 0; i < b->beams.size(); ++i) {
            bfs_status st = beam_stage1(b, static_cast<int>(i), d_inputs[i], b->plane, b->stats, b->ws, s);
            if (st != BFS_OK) return st;
        }
        return BFS_OK;
    }
    BFS_CUDA(cudaEventRecord(b->ev_fork, s));
    for (cudaStream_t t : b->lane_s) BFS_CUDA(cudaStreamWaitEvent(t, b->ev_fork, 0));
    for (size_t i = 0; i < b->beams.size(); ++i) {
        const int l = b->lane_of[i];
        bfs_status st = beam_stage1(b, static_cast<int>(i), d_inputs[i], b->lane_plane[l], b->lane_stats[l],
                                    b->lane_ws[l], b->lane_s[l]);
        if (st != BFS_OK) return st;
    }
    for (int l = 0; l < bfs_batch::kLanes; ++l) {
        BFS_CUDA(cudaEventRecord(b->ev_join[l], b->lane_s[l]));
        BFS_CUDA(cudaStreamWaitEvent(s, b->ev_join[l], 0));
    }
    return BFS_OK;
}

static bfs_status batch_stage2(bfs_batch* b, void* stream);

// Stage 1 of one run on s: replayed from the CUDA graph of the current
// buffer set when its inputs are the ones it was captured for (the first run
// is eager: kernel attributes are set then), else captured anew.
static bfs_status launch_stage1(bfs_batch* b, const float* const* d_inputs, cudaStream_t s) {
    const int nb = static_cast<int>(b->beams.size());
    bool same_inputs = b->exec && b->graph_inputs.size() == static_cast<size_t>(nb);
    for (int i = 0; same_inputs && i < nb; ++i) same_inputs = b->graph_inputs[i] == d_inputs[i];
    if (b->use_graph && b->runs >= 1 && !same_inputs) {
        if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
        if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
        cudaStream_t cs;
        BFS_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        bfs_status st = e == cudaSuccess ? enqueue_stage1(b, d_inputs, cs)
                                         : fail(BFS_ERR_CUDA, "begin capture: %s", cudaGetErrorString(e));
        cudaGraph_t g = nullptr;
        cudaError_t e2 = cudaStreamEndCapture(cs, &g);
        cudaStreamDestroy(cs);
        if (st != BFS_OK) { if (g) cudaGraphDestroy(g); return st; }
        if (e2 != cudaSuccess) return fail(BFS_ERR_CUDA, "end capture: %s", cudaGetErrorString(e2));
        b->graph = g;
        BFS_CUDA(cudaGraphInstantiate(&b->exec, g, 0));
        b->graph_inputs.assign(d_inputs, d_inputs + nb);
        same_inputs = true;
    }
    if (b->use_graph && b->exec && same_inputs) {
        BFS_CUDA(cudaGraphLaunch(b->exec, s));
    } else {
        bfs_status st = enqueue_stage1(b, d_inputs, s);
        if (st != BFS_OK) return st;
    }
    ++b->runs;
    return BFS_OK;
}

extern "C" bfs_status bfs_batch_run(bfs_batch* b, const float* const* d_inputs, void* stream) {
    BFS_ARG(b && d_inputs, "null argument");
    BFS_ARG(b->inflight == 0, "runs submitted with bfs_batch_submit are not collected yet");
    bfs_status st = launch_stage1(b, d_inputs, as_stream(stream));
    if (st != BFS_OK) return st;
    return batch_stage2(b, stream);
}

// ---- the asynchronous form --------------------------------------------------
// Makes buffer set k the one in the batch's stage-1 fields.
static void use_set(bfs_batch* b, int k) {
    if (b->active == k) return;
    std::swap(b->cands, b->cands_alt);
    std::swap(b->tags, b->tags_alt);
    std::swap(b->rec, b->rec_alt);
    std::swap(b->d_count, b->d_count_alt);
    std::swap(b->graph, b->graph_alt);
    std::swap(b->exec, b->exec_alt);
    std::swap(b->graph_inputs, b->graph_inputs_alt);
    b->active = k;
}

// The second buffer set, the stage-1 stream and the events (first submit).
static bfs_status ensure_async(bfs_batch* b) {
    if (b->s1) return BFS_OK;
    const size_t cap = b->capacity;
    BFS_CUDA(cudaMalloc(&b->cands_alt, cap * sizeof(bfs_cand)));
    if (!b->ordered) BFS_CUDA(cudaMalloc(&b->tags_alt, cap * sizeof(int)));
    if (b->ordered) BFS_CUDA(cudaMalloc(&b->rec_alt, sizeof(unsigned) * 2 * b->nrec));
    BFS_CUDA(cudaMalloc(&b->d_count_alt, sizeof(unsigned)));
    BFS_CUDA(cudaEventCreateWithFlags(&b->ev_in, cudaEventDisableTiming));
    for (auto& e : b->ev_done) BFS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    BFS_CUDA(cudaStreamCreateWithFlags(&b->s1, cudaStreamNonBlocking));
    return BFS_OK;
}

extern "C" bfs_status bfs_batch_submit(bfs_batch* b, const float* const* d_inputs, void* stream) {
    BFS_ARG(b && d_inputs, "null argument");
    BFS_ARG(b->inflight < 2, "two runs are in flight: collect one first");
    bfs_status st = ensure_async(b);
    if (st != BFS_OK) return st;
    const int k = b->next_set;
    use_set(b, k);
    // the inputs are ready once the caller's stream reaches this point
    BFS_CUDA(cudaEventRecord(b->ev_in, as_stream(stream)));
    BFS_CUDA(cudaStreamWaitEvent(b->s1, b->ev_in, 0));
    st = launch_stage1(b, d_inputs, b->s1);
    if (st != BFS_OK) return st;
    BFS_CUDA(cudaEventRecord(b->ev_done[k], b->s1));
    b->queue[(b->qhead + b->inflight) % 2] = k;
    ++b->inflight;
    b->next_set ^= 1;
    return BFS_OK;
}

extern "C" bfs_status bfs_batch_collect(bfs_batch* b, void* stream) {
    BFS_ARG(b != nullptr, "null argument");
    BFS_ARG(b->inflight > 0, "no submitted run to collect");
    const int k = b->queue[b->qhead];
    use_set(b, k);
    BFS_CUDA(cudaStreamWaitEvent(as_stream(stream), b->ev_done[k], 0));
    b->qhead ^= 1;
    --b->inflight;
    return batch_stage2(b, stream);
}

// Host-input form: beam i's input is copied from pinned host memory
// h_inputs[i] into d_inputs[i] on a copy stream while the compute stream
// runs beam i-1 (event dependencies), so the copies overlap the FDMT and
// search of the beams before them.  Copies and compute are captured together
// in one CUDA graph (after one eager run), replayed while the pointers stay
// the same.
static bfs_status enqueue_host_stage1(bfs_batch* b, const float* const* h_inputs,
                                      float* const* d_inputs, cudaStream_t cs, cudaStream_t cp) {
    const int nb = static_cast<int>(b->beams.size());
    BFS_CUDA(cudaMemsetAsync(b->d_count, 0, sizeof(unsigned), cs));
    BFS_CUDA(cudaEventRecord(b->events[nb], cs));
    BFS_CUDA(cudaStreamWaitEvent(cp, b->events[nb], 0));
    for (int i = 0; i < nb; ++i) {
        const bfs_fdmt_desc& d = b->beams[i];
        const size_t bytes = static_cast<size_t>(d.nchan) * d.ncols * sizeof(float);
        BFS_CUDA(cudaMemcpyAsync(d_inputs[i], h_inputs[i], bytes, cudaMemcpyHostToDevice, cp));
        BFS_CUDA(cudaEventRecord(b->events[i], cp));
        BFS_CUDA(cudaStreamWaitEvent(cs, b->events[i], 0));
        bfs_status st = beam_stage1(b, i, d_inputs[i], b->plane, b->stats, b->ws, cs);
        if (st != BFS_OK) return st;
    }
    // the copy stream joins the compute stream (required to end a capture)
    BFS_CUDA(cudaEventRecord(b->events[nb + 1], cp));
    BFS_CUDA(cudaStreamWaitEvent(cs, b->events[nb + 1], 0));
    return BFS_OK;
}

extern "C" bfs_status bfs_batch_run_host(bfs_batch* b, const float* const* h_inputs,
                                         float* const* d_inputs, void* stream) {
    BFS_ARG(b && h_inputs && d_inputs, "null argument");
    BFS_ARG(b->inflight == 0, "runs submitted with bfs_batch_submit are not collected yet");
    cudaStream_t s = as_stream(stream);
    const int nb = static_cast<int>(b->beams.size());
    for (int i = 0; i < nb; ++i) BFS_ARG(h_inputs[i] && d_inputs[i], "beam %d: null input pointer", i);
    if (b->events.empty()) {
        b->events.resize(nb + 2, nullptr);
        for (auto& e : b->events) BFS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    std::vector<const void*> ptrs;
    for (int i = 0; i < nb; ++i) ptrs.push_back(h_inputs[i]);
    for (int i = 0; i < nb; ++i) ptrs.push_back(d_inputs[i]);
    const bool same = b->hexec && ptrs == b->hgraph_ptrs;
    cudaStream_t cp;
    BFS_CUDA(cudaStreamCreateWithFlags(&cp, cudaStreamNonBlocking));
    bfs_status st = BFS_OK;
    if (same) {
        cudaError_t e = cudaGraphLaunch(b->hexec, s);
        if (e != cudaSuccess) st = fail(BFS_ERR_CUDA, "graph launch: %s", cudaGetErrorString(e));
    } else if (!b->use_graph || b->runs == 0) {
        st = enqueue_host_stage1(b, h_inputs, d_inputs, s, cp);  // eager (kernel set-up)
    } else {
        if (b->hexec) { cudaGraphExecDestroy(b->hexec); b->hexec = nullptr; }
        if (b->hgraph) { cudaGraphDestroy(b->hgraph); b->hgraph = nullptr; }
        cudaStream_t cs;
        BFS_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        st = e == cudaSuccess ? enqueue_host_stage1(b, h_inputs, d_inputs, cs, cp)
                              : fail(BFS_ERR_CUDA, "begin capture: %s", cudaGetErrorString(e));
        cudaGraph_t g = nullptr;
        cudaError_t e2 = cudaStreamEndCapture(cs, &g);
        cudaStreamDestroy(cs);
        if (st == BFS_OK && e2 != cudaSuccess) st = fail(BFS_ERR_CUDA, "end capture: %s", cudaGetErrorString(e2));
        if (st == BFS_OK) {
            b->hgraph = g;
            g = nullptr;
            e = cudaGraphInstantiate(&b->hexec, b->hgraph, 0);
            if (e != cudaSuccess) st = fail(BFS_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
        }
        if (g) cudaGraphDestroy(g);
        if (st == BFS_OK) {
            b->hgraph_ptrs = ptrs;
            e = cudaGraphLaunch(b->hexec, s);
            if (e != cudaSuccess) st = fail(BFS_ERR_CUDA, "graph launch: %s", cudaGetErrorString(e));
        }
    }
    cudaStreamDestroy(cp);
    if (st != BFS_OK) return st;
    ++b->runs;
    return batch_stage2(b, stream);
}

// ---- stage 2: all candidates at once --------------------------------------
static bfs_status batch_stage2(bfs_batch* b, void* stream) {
    cudaStream_t s = as_stream(stream);
    const int nb = static_cast<int>(b->beams.size());
    unsigned count = 0;
    BFS_CUDA(cudaMemcpyAsync(&count, b->d_count, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    BFS_CUDA(cudaStreamSynchronize(s));
    if (count > b->capacity)
        return fail(BFS_ERR_OVERFLOW, "%u candidates, batch capacity %u", count, b->capacity);
    b->n_cands = count;
    b->h_delegates.clear(); b->h_delegate_beam.clear(); b->h_delegate_size.clear();
    b->h_beam_first.assign(nb, 0); b->h_beam_count.assign(nb, 0); b->h_beam_cands.assign(nb, 0);
    b->n_groups = 0;
    if (count == 0) return BFS_OK;
    // canonical order (beam, row, sample, width)
    bfs_status st = b->ordered
        ? compact_ordered(b->cands, b->rec, b->rec + b->nrec, b->nrec, b->d_beam_rec, nb, b->sorted,
                          b->sorted_tags, s)
        : sort_tagged_candidates(b->cands, b->tags, count, b->max_rows, b->max_cols, nb - 1, b->widths_mode,
                                 b->param, b->sorted, b->sorted_tags, s);
    if (st != BFS_OK) return st;
    uint32_t ng = 0;
    st = bfs_cluster_grouped(b->sorted, count, b->sorted_tags, static_cast<uint32_t>(nb), b->metrics,
                             b->perm, b->offsets, b->delegates, &ng, stream);
    if (st != BFS_OK) return st;
    b->n_groups = ng;
    // delegates come back ordered by (mt, group); a stable sort by beam gives (beam, mt, group)
    const int bbits = std::max(1, bits_of(static_cast<unsigned long long>(nb)));
    size_t tb = 0;
    unsigned* nullu = nullptr;
    BFS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, nullu, nullu, nullu, nullu,
                                             static_cast<int>(ng), 0, bbits, s));
    int* inv = nullptr;
    unsigned* u = nullptr;   // key, key_sorted, val, order, beam_first (nb+1)
    bfs_cand* rec = nullptr; // rec, rec_out
    int* ints = nullptr;     // size, size_out, beam_out
    void* tmp = nullptr;
    st = stream_alloc(reinterpret_cast<void**>(&inv), sizeof(int) * count, s);
    if (st == BFS_OK) st = stream_alloc(reinterpret_cast<void**>(&u), sizeof(unsigned) * (4 * ng + nb + 1), s);
    if (st == BFS_OK) st = stream_alloc(reinterpret_cast<void**>(&rec), sizeof(bfs_cand) * 2 * ng, s);
    if (st == BFS_OK) st = stream_alloc(reinterpret_cast<void**>(&ints), sizeof(int) * 3 * ng, s);
    if (st == BFS_OK) st = stream_alloc(&tmp, tb ? tb : 16, s);
    if (st != BFS_OK) return st;
    unsigned *key = u, *key_sorted = u + ng, *val = u + 2 * ng, *order = u + 3 * ng, *bfirst = u + 4 * ng;
    const int th = 256;
    k_inverse_perm<<<static_cast<int>((count + th - 1) / th), th, 0, s>>>(b->perm, count, inv);
    BFS_LAUNCH_CHECK("k_inverse_perm");
    const int blg = static_cast<int>((ng + th - 1) / th);
    k_delegate_info<<<blg, th, 0, s>>>(b->sorted, b->sorted_tags, b->delegates, inv, b->offsets, ng, rec,
                                       ints, key, val);
    BFS_LAUNCH_CHECK("k_delegate_info");
    BFS_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, key, key_sorted, val, order, static_cast<int>(ng), 0,
                                             bbits, s));
    k_permute_delegates<<<blg, th, 0, s>>>(rec, ints, key_sorted, order, ng, rec + ng, ints + ng,
                                           ints + 2 * ng);
    BFS_LAUNCH_CHECK("k_permute_delegates");
    k_beam_bounds<<<(nb + 1 + th - 1) / th, th, 0, s>>>(b->sorted_tags, count, nb, bfirst);
    BFS_LAUNCH_CHECK("k_beam_bounds");
    b->h_delegates.resize(ng);
    b->h_delegate_size.resize(ng);
    b->h_delegate_beam.resize(ng);
    std::vector<unsigned> first(nb + 1);
    BFS_CUDA(cudaMemcpyAsync(b->h_delegates.data(), rec + ng, sizeof(bfs_cand) * ng, cudaMemcpyDeviceToHost, s));
    BFS_CUDA(cudaMemcpyAsync(b->h_delegate_size.data(), ints + ng, sizeof(int) * ng, cudaMemcpyDeviceToHost, s));
    BFS_CUDA(cudaMemcpyAsync(b->h_delegate_beam.data(), ints + 2 * ng, sizeof(int) * ng, cudaMemcpyDeviceToHost, s));
    BFS_CUDA(cudaMemcpyAsync(first.data(), bfirst, sizeof(unsigned) * (nb + 1), cudaMemcpyDeviceToHost, s));
    cudaFreeAsync(inv, s);
    cudaFreeAsync(u, s);
    cudaFreeAsync(rec, s);
    cudaFreeAsync(ints, s);
    cudaFreeAsync(tmp, s);
    BFS_CUDA(cudaStreamSynchronize(s));
    for (int i = 0; i < nb; ++i) b->h_beam_cands[i] = static_cast<int>(first[i + 1] - first[i]);
    for (uint32_t i = 0; i < ng; ++i) {
        const int beam = b->h_delegate_beam[i];
        if (b->h_beam_count[beam] == 0) b->h_beam_first[beam] = static_cast<int>(i);
        ++b->h_beam_count[beam];
    }
    return BFS_OK;
}

extern "C" bfs_status bfs_batch_counts(const bfs_batch* b, uint32_t* n_cands, uint32_t* n_groups) {
    BFS_ARG(b != nullptr, "null argument");
    if (n_cands) *n_cands = b->n_cands;
    if (n_groups) *n_groups = b->n_groups;
    return BFS_OK;
}

extern "C" bfs_status bfs_batch_beam_results(const bfs_batch* b, int beam, bfs_cand* delegates,
                                             int* group_sizes, int cap, int* n_delegates,
                                             uint32_t* n_candidates) {
    BFS_ARG(b != nullptr && beam >= 0 && beam < static_cast<int>(b->beams.size()), "bad beam");
    const int n = b->h_beam_count.empty() ? 0 : b->h_beam_count[beam];
    if (n_delegates) *n_delegates = n;
    if (n_candidates) *n_candidates = b->h_beam_cands.empty() ? 0u : static_cast<uint32_t>(b->h_beam_cands[beam]);
    const int first = n ? b->h_beam_first[beam] : 0;
    for (int i = 0; i < n && i < cap; ++i) {
        if (delegates) delegates[i] = b->h_delegates[first + i];
        if (group_sizes) group_sizes[i] = b->h_delegate_size[first + i];
    }
    return BFS_OK;
}
