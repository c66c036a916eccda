// The FDMT plan object behind the opaque bfs_fdmt_plan handle (shared by the
// forward and adjoint translation units).
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "internal.h"

struct bfs_fdmt_plan {
    bfs::FdmtPlanHost host;
    int device = -1;
    bool host_only = false;
    bool external_ws = false;
    int fuse_depth = 0;
    int precision = BFS_PREC_F32;      // storage of the planes between levels
    int4* d_tab = nullptr;             // per level, per output row: {a, b, shift, exps}
    std::vector<size_t> tab_off;       // offset of each level's table in d_tab
    void* d_buf[2] = {nullptr, nullptr};
    size_t buf_rows[2] = {0, 0};
    size_t ws_bytes = 0;
    bfs::HeadPlan head;                     // fused levels 0..k (depth 0 = not used)
    bfs::HeadGroup* d_head_groups = nullptr;
    int* d_head_tab = nullptr;
    // passes after the head (or level 0): a fused segment of levels l0+1..l1
    // (tiles non-empty) or one plain merge level (l1 = l0 + 1, no tiles)
    std::vector<bfs::SegPlan> passes;
    std::vector<int> plane_buf;        // per level: ping-pong plane holding it in HBM (-1: never)
    bfs::SegTile* d_seg_tiles = nullptr;  // every fused segment's tiles, concatenated
    int* d_seg_ent = nullptr;          // every fused segment's entries, concatenated
    std::vector<size_t> seg_tile0, seg_ent0;  // per pass: offsets into the two arrays
    int* d_lvl0 = nullptr;             // Pravir plans: level-0 row cumsum (nchan+1) then delays
    int* d_ones_tau = nullptr;         // FDMT of 0/1 rows: tau [out_row][channel] (first use)
    int ones_max_tau = -1;
    // adjoint (built on the first adjoint call): per level l >= 1, for every
    // row of level l-1 the level-l rows that read it, as CSR {row, shift}
    bfs::AdjointTables adj;
    int* d_adj_off = nullptr;
    int2* d_adj_ent = nullptr;
    void* d_adj_buf[2] = {nullptr, nullptr};  // plan-owned adjoint planes (bfs_fdmt_adjoint)
    ~bfs_fdmt_plan() {
        if (d_tab) cudaFree(d_tab);
        if (d_head_groups) cudaFree(d_head_groups);
        if (d_head_tab) cudaFree(d_head_tab);
        if (d_lvl0) cudaFree(d_lvl0);
        if (d_seg_tiles) cudaFree(d_seg_tiles);
        if (d_seg_ent) cudaFree(d_seg_ent);
        if (d_ones_tau) cudaFree(d_ones_tau);
        for (void* b : d_buf)
            if (b) cudaFree(b);
        if (d_adj_off) cudaFree(d_adj_off);
        if (d_adj_ent) cudaFree(d_adj_ent);
        for (void* b : d_adj_buf)
            if (b) cudaFree(b);
    }
};
