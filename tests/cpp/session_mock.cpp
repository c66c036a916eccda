// Test double for running tests/cpp/session_demo.cpp on a machine without a
// GPU: linked into the demo executable, whose own definitions take
// precedence over the library's. It stands in for the CUDA runtime calls
// the drop-in header makes (device memory is host memory) and for the
// GPU-side C-ABI entries:
//   - the chunk, whose planes are a fixed function of the raw chunk;
//   - the boxcar gather: one candidate per row at its largest sample;
//   - the clustering: every candidate a group of its own;
//   - the streaming reader: host reads through bfs_guppi_read_chunk.
// The GUPPI file index, the session geometry and the coherent-DM grid come
// from the real library.  The session's control flow (chunk order, buffer
// sizes, images, log) is what the test checks; nothing here runs a kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "bfs.h"

extern "C" {

cudaError_t cudaMalloc(void** p, size_t n) {
    *p = std::malloc(n ? n : 1);
    return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
cudaError_t cudaFree(void* p) {
    std::free(p);
    return cudaSuccess;
}
cudaError_t cudaMemcpy(void* dst, const void* src, size_t n, cudaMemcpyKind) {
    std::memcpy(dst, src, n);
    return cudaSuccess;
}

}  // extern "C"

struct bfs_chunk {
    bfs_chunk_desc d;
    int64_t mbin, nov_pc, mbin_adj, msamp, rows, len_chunk, cplx, max_dt;
};

struct bfs_guppi_reader {
    const bfs_guppi_file* f;
    int64_t len, ov;
    int block = 0;
    int64_t chunk = 0;
    std::vector<int8_t> host;
};

extern "C" {

bfs_status bfs_chunk_create(const bfs_chunk_desc* d, bfs_chunk** out) {
    if (d->nbin % d->len_sft != 0) return BFS_ERR_ARG;
    bfs_chunk* c = new bfs_chunk;
    c->d = *d;
    c->mbin = d->nbin / d->len_sft;
    c->nov_pc = d->noverlap / d->len_sft;
    c->mbin_adj = c->mbin - 2 * c->nov_pc;
    c->msamp = static_cast<int64_t>(d->nfft) * c->mbin_adj;
    c->rows = static_cast<int64_t>(d->nchan) * d->len_sft;
    c->len_chunk = static_cast<int64_t>(d->nbin - 2 * d->noverlap) * d->nfft;
    c->cplx = static_cast<int64_t>(d->npol / 2) * d->nfft * d->nchan * d->nbin;
    c->max_dt = d->max_dt ? d->max_dt : d->len_sft;
    *out = c;
    return BFS_OK;
}
bfs_status bfs_chunk_destroy(bfs_chunk* c) {
    delete c;
    return BFS_OK;
}
bfs_status bfs_chunk_info(const bfs_chunk* c, int64_t* info, int cap) {
    const int64_t v[8] = {c->mbin, c->nov_pc, c->mbin_adj, c->msamp, c->rows, c->len_chunk, c->cplx, c->max_dt};
    for (int i = 0; i < cap && i < 8; ++i) info[i] = v[i];
    return BFS_OK;
}

// plane i (coherent DM), row r, sample t = (s + 7 i + 3 r + t) % 97 with s the
// byte sum of the raw chunk
bfs_status bfs_chunk_process_raw(bfs_chunk* c, const int8_t* d_raw, void* d_spec, const double*, int ndm,
                                 float* d_out, void*) {
    const int64_t raw = static_cast<int64_t>(c->d.nchan) * c->len_chunk * c->d.npol;
    int64_t s = 0;
    for (int64_t k = 0; k < raw; ++k) s += d_raw[k];
    std::memset(d_spec, 0, static_cast<size_t>(c->cplx) * 8);  // the spectra are written
    for (int i = 0; i < ndm; ++i)
        for (int64_t r = 0; r < c->max_dt; ++r)
            for (int64_t t = 0; t < c->msamp; ++t)
                d_out[(i * c->max_dt + r) * c->msamp + t] =
                    static_cast<float>((((s + 7 * i + 3 * r + t) % 97) + 97) % 97);
    return BFS_OK;
}

bfs_status bfs_boxcar_gather(const float* plane, int rows, int cols, const float*, float, const float*, int,
                             int, int, bfs_cand* out, uint32_t capacity, uint32_t* h_count, void*) {
    *h_count = static_cast<uint32_t>(rows);
    for (int r = 0; r < rows && static_cast<uint32_t>(r) < capacity; ++r) {
        const float* p = plane + static_cast<size_t>(r) * cols;
        const int t = static_cast<int>(std::max_element(p, p + cols) - p);
        out[r] = bfs_cand{t, r, 1, p[t]};
    }
    return static_cast<uint32_t>(rows) > capacity ? BFS_ERR_OVERFLOW : BFS_OK;
}

bfs_status bfs_cluster(const bfs_cand* c, uint32_t n, const int*, int* perm, int* offsets, int* delegates,
                       uint32_t* h_ngroups, void*) {
    std::vector<int> idx(n);
    for (uint32_t i = 0; i < n; ++i) idx[i] = static_cast<int>(i);
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return c[a].mt < c[b].mt; });
    for (uint32_t i = 0; i < n; ++i) {
        perm[i] = static_cast<int>(i);
        offsets[i] = static_cast<int>(i);
        delegates[i] = idx[i];
    }
    offsets[n] = static_cast<int>(n);
    *h_ngroups = n;
    return BFS_OK;
}

bfs_status bfs_guppi_reader_create(const bfs_guppi_file* f, int64_t len, int64_t ov, int, int,
                                   bfs_guppi_reader** out) {
    bfs_guppi_reader* r = new bfs_guppi_reader;
    r->f = f;
    r->len = len;
    r->ov = ov;
    bfs_guppi_header h{};
    bfs_guppi_block_header(f, 0, &h);
    r->host.resize(static_cast<size_t>(h.nchan) * len * h.npol);
    *out = r;
    return BFS_OK;
}
bfs_status bfs_guppi_reader_destroy(bfs_guppi_reader* r) {
    delete r;
    return BFS_OK;
}
bfs_status bfs_guppi_reader_next(bfs_guppi_reader* r, void* d_dst, void*, const int8_t** h_src, int* block,
                                 int64_t* chunk) {
    int nb = 0;
    bfs_guppi_blocks(r->f, &nb);
    for (;;) {
        if (r->block >= nb) {
            *block = -1;
            return BFS_OK;
        }
        int64_t n = 0;
        bfs_guppi_chunk_count(r->f, r->block, r->len, r->ov, &n);
        if (r->chunk < n) break;
        ++r->block;
        r->chunk = 0;
    }
    const bfs_status st = bfs_guppi_read_chunk(r->f, r->block, r->chunk, r->len, r->ov, r->host.data(),
                                               r->host.size());
    if (st != BFS_OK) return st;
    if (d_dst) std::memcpy(d_dst, r->host.data(), r->host.size());
    if (h_src) *h_src = r->host.data();
    *block = r->block;
    if (chunk) *chunk = r->chunk;
    ++r->chunk;
    return BFS_OK;
}

}  // extern "C"
