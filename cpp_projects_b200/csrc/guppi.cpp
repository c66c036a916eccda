// GUPPI RAW session input: header cards, block index, per-channel strided
// chunk reads with overlap, and a streaming reader that fills pinned host
// buffers on a background thread and copies them to the device on the
// caller's stream.
//
// Reference: CSession_guppi / CTelescopeHeader (MyVSLib_C++/CDMT/
// Session_guppi.cpp:31-85 block count, :111-283 header, :336-369 chunk
// download; MyVSLib_C++/TelescopeHeader.cpp:88-124,175-347; SessionB.cpp:
// 226-273 chunk loop; SessionB.h:128-140 byte counts).
//
// Header: 80-byte "KEY     = value" cards.  As the reference: the block is
// accepted when "RAW" occurs in the header and the keys DIRECTIO, NBITS,
// CHAN_BW, OBSFREQ, OBSNCHAN, OBSBW, BLOCSIZE, TELESCOP (GBT or PARKES), NPOL
// and TBIN are present (value from column 9 of the key, TBIN from column
// 10); the data start after the third "END" in the header text (the END
// card of GUPPI headers, whose BACKEND key holds the first), rounded up to a
// multiple of 512 bytes when DIRECTIO is non-zero, as is the data length of
// every block.  A negative CHAN_BW means the channels are stored in
// descending frequency; chunks are returned in ascending frequency.
//
// Block data: [nchan][nsamp][npol * nbits / 8] bytes.  Chunk j of a block
// covers samples j * (len - 2 ov) .. + len of every channel; the last chunk
// of a block ends at the block's last sample.  (The reference rewinds the
// file by a whole chunk before reading the last chunk of a block, which
// reads before the block's data when a block holds one chunk; that step is
// not reproduced.)
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "internal.h"

namespace {

constexpr size_t kHeaderScan = 10000;  // bytes the reference reads for a header

const char* find(const char* hay, size_t n, const char* needle) {
    const size_t m = std::strlen(needle);
    if (m == 0 || n < m) return nullptr;
    for (size_t i = 0; i + m <= n; ++i)
        if (std::memcmp(hay + i, needle, m) == 0) return hay + i;
    return nullptr;
}

}  // namespace

struct bfs_guppi_file {
    std::string path;
    std::vector<bfs_guppi_header> blocks;   // every block's header (data_offset absolute)
};

namespace bfs {

// Parses one header from text (len bytes; the header must fit).  Sets the
// data offset relative to the start of the text.
static bfs_status parse_guppi_header(const char* text, size_t len, bfs_guppi_header* h) {
    *h = bfs_guppi_header{};
    const size_t n = std::min(len, kHeaderScan);
    BFS_ARG(find(text, n, "RAW") != nullptr, "not a RAW header");
    const char* pend = text;
    for (int i = 0; i < 3; ++i) {
        const char* q = find(pend, n - static_cast<size_t>(pend - text), "END");
        BFS_ARG(q != nullptr, "header has fewer than three \"END\"");
        pend = q + 1;
    }
    int64_t off = static_cast<int64_t>(pend - 1 - text) + 3;
    auto value = [&](const char* key, int col, std::string* out) -> bool {
        const char* p = find(text, n, key);
        if (!p) return false;
        const char* v = p + col;
        const char* e = text + n;
        size_t k = 0;
        while (v + k < e && v[k] != '\0' && k < 71) ++k;
        out->assign(v, k);
        return true;
    };
    std::string s;
    BFS_ARG(value("DIRECTIO", 9, &s), "header has no DIRECTIO");
    h->directio = std::atoi(s.c_str()) != 0;
    if (h->directio) off = (off + 511) / 512 * 512;
    h->data_offset = off;
    BFS_ARG(value("NBITS", 9, &s), "header has no NBITS");
    h->nbits = std::atoi(s.c_str());
    BFS_ARG(value("CHAN_BW", 9, &s), "header has no CHAN_BW");
    const float chan_bw = static_cast<float>(std::atof(s.c_str()));
    h->straight_order = chan_bw >= 0.0f;
    h->chan_bw = std::fabs(chan_bw);
    BFS_ARG(value("OBSFREQ", 9, &s), "header has no OBSFREQ");
    h->obsfreq = std::fabs(static_cast<float>(std::atof(s.c_str())));
    BFS_ARG(value("OBSNCHAN", 9, &s), "header has no OBSNCHAN");
    h->nchan = std::atoi(s.c_str());
    BFS_ARG(value("OBSBW", 9, &s), "header has no OBSBW");
    h->obsbw = std::fabs(static_cast<float>(std::atof(s.c_str())));
    BFS_ARG(value("BLOCSIZE", 9, &s), "header has no BLOCSIZE");
    h->blocsize = std::atoi(s.c_str());
    BFS_ARG(value("TELESCOP", 9, &s), "header has no TELESCOP");
    {
        const size_t g = s.find("GBT"), pk = s.find("PARKES");
        if (g != std::string::npos) {
            BFS_ARG(g <= 20, "TELESCOP value not recognised");
            h->telescope = BFS_GUPPI_GBT;
        } else {
            BFS_ARG(pk != std::string::npos && pk <= 20, "TELESCOP is neither GBT nor PARKES");
            h->telescope = BFS_GUPPI_PARKES;
        }
    }
    BFS_ARG(value("NPOL", 9, &s), "header has no NPOL");
    h->npol = std::atoi(s.c_str());
    BFS_ARG(value("TBIN", 10, &s), "header has no TBIN");
    h->tbin = static_cast<float>(std::atof(s.c_str()));
    BFS_ARG(h->nbits == 8, "NBITS %d: only 8-bit samples are supported", h->nbits);
    BFS_ARG(h->nchan >= 1 && h->npol >= 1 && h->blocsize > 0, "bad header sizes");
    BFS_ARG(h->blocsize % (static_cast<int64_t>(h->nchan) * h->npol) == 0,
            "BLOCSIZE %lld is not a whole number of samples per channel", static_cast<long long>(h->blocsize));
    h->nsamp = h->blocsize / (static_cast<int64_t>(h->nchan) * h->npol);
    h->fmin = h->obsfreq - h->obsbw / 2.0f;
    h->fmax = h->obsfreq + h->obsbw / 2.0f;
    return BFS_OK;
}

static int64_t padded(const bfs_guppi_header& h, int64_t v) {
    return h.directio ? (v + 511) / 512 * 512 : v;
}

static int64_t chunk_count(const bfs_guppi_header& h, int64_t len, int64_t ov) {
    if (len <= 2 * ov || h.nsamp < len) return 0;
    return (h.nsamp - 2 * ov - 1) / (len - 2 * ov) + 1;
}

static int64_t chunk_start(const bfs_guppi_header& h, int64_t j, int64_t n, int64_t len, int64_t ov) {
    return j == n - 1 ? h.nsamp - len : j * (len - 2 * ov);
}

// Reads chunk j of one block into dst [nchan][len][npol] (ascending frequency).
static bfs_status read_chunk(FILE* f, const bfs_guppi_header& h, int64_t j, int64_t len, int64_t ov,
                             int8_t* dst) {
    const int64_t n = chunk_count(h, len, ov);
    BFS_ARG(j >= 0 && j < n, "chunk %lld out of range (%lld chunks)", static_cast<long long>(j),
            static_cast<long long>(n));
    const int64_t s0 = chunk_start(h, j, n, len, ov);
    const int64_t bps = h.npol;  // bytes per sample per channel (8-bit)
    const int64_t chan_bytes = h.nsamp * bps;
    for (int c = 0; c < h.nchan; ++c) {
        const int64_t pos = h.data_offset + c * chan_bytes + s0 * bps;
        const int slot = h.straight_order ? c : h.nchan - 1 - c;
        int8_t* out = dst + static_cast<int64_t>(slot) * len * bps;
        if (std::fseek(f, static_cast<long>(pos), SEEK_SET) != 0)
            return fail(BFS_ERR_ARG, "seek to %lld failed", static_cast<long long>(pos));
        const size_t got = std::fread(out, 1, static_cast<size_t>(len * bps), f);
        BFS_ARG(got == static_cast<size_t>(len * bps), "file ends inside block data");
    }
    return BFS_OK;
}

}  // namespace bfs

using namespace bfs;

extern "C" bfs_status bfs_guppi_parse_header(const char* text, size_t len, bfs_guppi_header* out) {
    BFS_ARG(text != nullptr && out != nullptr, "null argument");
    return parse_guppi_header(text, len, out);
}

extern "C" bfs_status bfs_guppi_open(const char* path, bfs_guppi_file** out) {
    BFS_ARG(path != nullptr && out != nullptr, "null argument");
    *out = nullptr;
    std::unique_ptr<FILE, int (*)(FILE*)> f(std::fopen(path, "rb"), &std::fclose);
    BFS_ARG(f != nullptr, "cannot open %s", path);
    std::unique_ptr<bfs_guppi_file> g(new bfs_guppi_file);
    g->path = path;
    std::vector<char> buf(kHeaderScan);
    int64_t pos = 0;
    for (;;) {
        if (std::fseek(f.get(), static_cast<long>(pos), SEEK_SET) != 0) break;
        const size_t got = std::fread(buf.data(), 1, buf.size(), f.get());
        if (got == 0) break;
        bfs_guppi_header h{};
        if (parse_guppi_header(buf.data(), got, &h) != BFS_OK) break;
        h.data_offset += pos;
        // the block's data must be in the file
        if (std::fseek(f.get(), 0, SEEK_END) != 0) break;
        const long end = std::ftell(f.get());
        if (h.data_offset + h.blocsize > end) break;
        g->blocks.push_back(h);
        pos = h.data_offset + padded(h, h.blocsize);
    }
    BFS_ARG(!g->blocks.empty(), "%s holds no readable GUPPI block", path);
    *out = g.release();
    return BFS_OK;
}

extern "C" bfs_status bfs_guppi_close(bfs_guppi_file* g) {
    delete g;
    return BFS_OK;
}

extern "C" bfs_status bfs_guppi_blocks(const bfs_guppi_file* g, int* nblocks) {
    BFS_ARG(g != nullptr && nblocks != nullptr, "null argument");
    *nblocks = static_cast<int>(g->blocks.size());
    return BFS_OK;
}

extern "C" bfs_status bfs_guppi_block_header(const bfs_guppi_file* g, int block, bfs_guppi_header* out) {
    BFS_ARG(g != nullptr && out != nullptr, "null argument");
    BFS_ARG(block >= 0 && block < static_cast<int>(g->blocks.size()), "block %d out of range", block);
    *out = g->blocks[block];
    return BFS_OK;
}

extern "C" bfs_status bfs_guppi_chunk_count(const bfs_guppi_file* g, int block, int64_t len_chunk,
                                            int64_t noverlap, int64_t* nchunks) {
    BFS_ARG(g != nullptr && nchunks != nullptr, "null argument");
    BFS_ARG(block >= 0 && block < static_cast<int>(g->blocks.size()), "block %d out of range", block);
    BFS_ARG(len_chunk > 2 * noverlap && noverlap >= 0, "need len_chunk > 2 * noverlap >= 0");
    *nchunks = chunk_count(g->blocks[block], len_chunk, noverlap);
    return BFS_OK;
}

extern "C" bfs_status bfs_guppi_read_chunk(const bfs_guppi_file* g, int block, int64_t chunk,
                                           int64_t len_chunk, int64_t noverlap, int8_t* dst,
                                           size_t dst_bytes) {
    BFS_ARG(g != nullptr && dst != nullptr, "null argument");
    BFS_ARG(block >= 0 && block < static_cast<int>(g->blocks.size()), "block %d out of range", block);
    BFS_ARG(len_chunk > 2 * noverlap && noverlap >= 0, "need len_chunk > 2 * noverlap >= 0");
    const bfs_guppi_header& h = g->blocks[block];
    BFS_ARG(dst_bytes >= static_cast<size_t>(h.nchan) * len_chunk * h.npol,
            "dst holds %zu bytes, the chunk needs %lld", dst_bytes,
            static_cast<long long>(h.nchan) * len_chunk * h.npol);
    std::unique_ptr<FILE, int (*)(FILE*)> f(std::fopen(g->path.c_str(), "rb"), &std::fclose);
    BFS_ARG(f != nullptr, "cannot open %s", g->path.c_str());
    return read_chunk(f.get(), h, chunk, len_chunk, noverlap, dst);
}

// ---------------------------------------------------------------------------
// Streaming reader: a background thread reads the chunks of every block in
// order into `nbuf` pinned host buffers; bfs_guppi_reader_next hands the
// next filled buffer to the caller (and, given a device pointer, copies it
// there on the caller's stream).  A buffer goes back to the reader once the
// copy that read it has completed (an event on that stream), so host reads,
// H2D copies and the caller's kernels overlap.
// ---------------------------------------------------------------------------
struct bfs_guppi_reader {
    const bfs_guppi_file* g = nullptr;
    int64_t len = 0, ov = 0;
    size_t bytes = 0;
    struct Slot {
        int8_t* host = nullptr;
        cudaEvent_t done = nullptr;  // recorded after the copy that reads `host`
        bool copy_pending = false;
        int block = -1;
        int64_t chunk = -1;
        bfs_status st = BFS_OK;
        std::string err;
    };
    std::vector<Slot> slots;
    std::deque<int> free_q, full_q;
    std::mutex mu;
    std::condition_variable cv;
    std::thread worker;
    bool stop = false, finished = false;
    bool pinned = true;
    int last = -1;  // slot handed out by the previous next() call

    ~bfs_guppi_reader() {
        {
            std::lock_guard<std::mutex> lock(mu);
            stop = true;
        }
        cv.notify_all();
        if (worker.joinable()) worker.join();
        for (Slot& s : slots) {
            if (s.done) {
                cudaEventSynchronize(s.done);
                cudaEventDestroy(s.done);
            }
            if (s.host) {
                if (pinned) cudaFreeHost(s.host);
                else std::free(s.host);
            }
        }
    }

    void run() {
        std::unique_ptr<FILE, int (*)(FILE*)> f(std::fopen(g->path.c_str(), "rb"), &std::fclose);
        for (size_t b = 0; b < g->blocks.size(); ++b) {
            const bfs_guppi_header& h = g->blocks[b];
            const int64_t n = chunk_count(h, len, ov);
            for (int64_t j = 0; j < n; ++j) {
                int id;
                {
                    std::unique_lock<std::mutex> lock(mu);
                    cv.wait(lock, [&] { return stop || !free_q.empty(); });
                    if (stop) return;
                    id = free_q.front();
                    free_q.pop_front();
                }
                Slot& s = slots[id];
                if (s.copy_pending) {  // the previous copy out of this buffer must be done
                    cudaEventSynchronize(s.done);
                    s.copy_pending = false;
                }
                s.block = static_cast<int>(b);
                s.chunk = j;
                s.st = f ? read_chunk(f.get(), h, j, len, ov, s.host) : BFS_ERR_ARG;
                if (s.st != BFS_OK) s.err = bfs_last_error();
                {
                    std::lock_guard<std::mutex> lock(mu);
                    full_q.push_back(id);
                }
                cv.notify_all();
                if (s.st != BFS_OK) {
                    std::lock_guard<std::mutex> lock(mu);
                    finished = true;
                    cv.notify_all();
                    return;
                }
            }
        }
        std::lock_guard<std::mutex> lock(mu);
        finished = true;
        cv.notify_all();
    }
};

extern "C" bfs_status bfs_guppi_reader_create(const bfs_guppi_file* g, int64_t len_chunk, int64_t noverlap,
                                              int nbuffers, int pinned, bfs_guppi_reader** out) {
    BFS_ARG(g != nullptr && out != nullptr, "null argument");
    BFS_ARG(len_chunk > 2 * noverlap && noverlap >= 0, "need len_chunk > 2 * noverlap >= 0");
    BFS_ARG(nbuffers >= 1 && nbuffers <= 16, "nbuffers must be in 1..16");
    *out = nullptr;
    const bfs_guppi_header& h0 = g->blocks[0];
    for (const bfs_guppi_header& h : g->blocks)
        BFS_ARG(h.nchan == h0.nchan && h.npol == h0.npol, "blocks differ in channels or polarisations");
    std::unique_ptr<bfs_guppi_reader> r(new bfs_guppi_reader);
    r->g = g;
    r->len = len_chunk;
    r->ov = noverlap;
    r->pinned = pinned != 0;
    r->bytes = static_cast<size_t>(h0.nchan) * len_chunk * h0.npol;
    r->slots.resize(nbuffers);
    for (int i = 0; i < nbuffers; ++i) {
        auto& s = r->slots[i];
        if (r->pinned) {
            BFS_CUDA(cudaMallocHost(reinterpret_cast<void**>(&s.host), r->bytes));
            BFS_CUDA(cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming));
        } else {
            s.host = static_cast<int8_t*>(std::malloc(r->bytes));
            BFS_ARG(s.host != nullptr, "out of host memory");
        }
        r->free_q.push_back(i);
    }
    r->worker = std::thread([p = r.get()] { p->run(); });
    *out = r.release();
    return BFS_OK;
}

extern "C" bfs_status bfs_guppi_reader_destroy(bfs_guppi_reader* r) {
    delete r;
    return BFS_OK;
}

// Next chunk: *block = -1 when the file is exhausted.  With d_dst non-null
// (a device buffer of the chunk's size, pinned reader) the chunk is copied
// there asynchronously on `stream`; *h_src (optional) points at the host
// copy, valid until the next call.
extern "C" bfs_status bfs_guppi_reader_next(bfs_guppi_reader* r, void* d_dst, void* stream,
                                            const int8_t** h_src, int* block, int64_t* chunk) {
    BFS_ARG(r != nullptr && block != nullptr, "null argument");
    BFS_ARG(d_dst == nullptr || r->pinned, "device copies need a pinned reader");
    // the buffer handed out last time goes back to the reader
    if (r->last >= 0) {
        {
            std::lock_guard<std::mutex> lock(r->mu);
            r->free_q.push_back(r->last);
        }
        r->cv.notify_all();
        r->last = -1;
    }
    int id;
    {
        std::unique_lock<std::mutex> lock(r->mu);
        r->cv.wait(lock, [&] { return !r->full_q.empty() || r->finished; });
        if (r->full_q.empty()) {
            *block = -1;
            if (chunk) *chunk = -1;
            if (h_src) *h_src = nullptr;
            return BFS_OK;
        }
        id = r->full_q.front();
        r->full_q.pop_front();
    }
    auto& s = r->slots[id];
    if (s.st != BFS_OK) return fail(s.st, "%s", s.err.c_str());
    *block = s.block;
    if (chunk) *chunk = s.chunk;
    if (h_src) *h_src = s.host;
    if (d_dst) {
        cudaStream_t st = as_stream(stream);
        BFS_CUDA(cudaMemcpyAsync(d_dst, s.host, r->bytes, cudaMemcpyHostToDevice, st));
        BFS_CUDA(cudaEventRecord(s.done, st));
        s.copy_pending = true;
    }
    r->last = id;
    return BFS_OK;
}

// ---------------------------------------------------------------------------
// Session geometry (CSessionB::launch, MyVSLib_C++/CDMT/SessionB.cpp:144-160
// and 184-206, with get_optimal_overlap :384-392 and get_coherent_dms
// :395-401).  The arithmetic keeps the reference's types: float header
// fields and float products, double dispersion constants, C rounding.
// ---------------------------------------------------------------------------
namespace {

constexpr double kDispersion = 4.148808e3;  // MHz^2 pc^-1 cm^3 s, the session's constant

// Dispersion delay (s) between f_lo and f_hi at dm: the squares are float
// products, the reciprocals and the rest double, the result stored as float.
float session_delay(double dm, float f_lo, float f_hi) {
    const float lo2 = f_lo * f_lo;
    const float hi2 = f_hi * f_hi;
    return static_cast<float>(kDispersion * dm * (1.0 / static_cast<double>(lo2) - 1.0 / static_cast<double>(hi2)));
}

}  // namespace

extern "C" bfs_status bfs_guppi_session_plan(const bfs_guppi_header* h, float pulse_length, double d_min,
                                             double d_max, int nbin, int nfft, bfs_guppi_session* out) {
    BFS_ARG(h != nullptr && out != nullptr, "null argument");
    *out = bfs_guppi_session{};
    BFS_ARG(std::isfinite(pulse_length) && pulse_length > 0.0f, "pulse length must be positive");
    BFS_ARG(std::isfinite(h->tbin) && h->tbin > 0.0f, "TBIN must be positive");
    BFS_ARG(h->nchan >= 1 && h->obsbw > 0.0f && std::isfinite(h->obsbw), "bad band in the header");
    BFS_ARG(nbin >= 2 && nfft >= 1, "need nbin >= 2 and nfft >= 1");
    BFS_ARG(std::isfinite(d_max) && d_max > 0.0 && std::isfinite(d_min), "need a positive finite d_max");
    const float fmin = static_cast<float>(static_cast<double>(h->obsfreq) - std::fabs(h->obsbw) / 2.0);
    const float fmax = static_cast<float>(static_cast<double>(h->obsfreq) + std::fabs(h->obsbw) / 2.0);
    BFS_ARG(fmin > 0.0f && fmax > fmin, "band edges %g..%g MHz", fmin, fmax);
    BFS_ARG(static_cast<float>(d_min) <= static_cast<float>(d_max), "d_min above d_max");

    // fine channels per coarse channel: the pulse length in samples
    const float np = std::ceil(pulse_length / h->tbin);
    BFS_ARG(np >= 1.0f && np <= 1048576.0f, "pulse length gives %g fine channels", np);
    const int len_sft = static_cast<int>(np);

    // overlap: half the delay across the lowest fine channel at d_max,
    // rounded to a power of two
    const float bw_chan = std::fabs(h->obsbw) / static_cast<float>(h->nchan * len_sft);
    const float f_top = fmin + bw_chan;
    const float delay_samples = std::round(session_delay(d_max, fmin, f_top) / h->tbin);
    BFS_ARG(std::isfinite(delay_samples) && delay_samples >= 0.0f && delay_samples < 2147483648.0f,
            "overlap of %g samples", delay_samples);
    const int optimal = static_cast<int>(delay_samples);
    const int half = optimal / 2;
    const int noverlap = half > 0 ? static_cast<int>(std::pow(2.0, std::round(std::log2(static_cast<double>(half)))))
                                  : 0;
    BFS_ARG(2LL * noverlap < nbin, "nbin must be greater than %d", 2 * noverlap);

    // coherent DMs: the whole band's delay at d_max in units of t_p^2 / tbin
    const float t_d = session_delay(d_max, fmin, fmax);
    const float ncoh = std::ceil(t_d * h->tbin / (pulse_length * pulse_length));
    BFS_ARG(ncoh >= 1.0f && ncoh <= 1048576.0f, "%g coherent DMs", ncoh);

    out->len_sft = len_sft;
    out->noverlap = noverlap;
    out->len_chunk = static_cast<int64_t>(nbin - 2 * noverlap) * nfft;
    out->ncoherent = static_cast<int>(ncoh);
    out->optimal_overlap = optimal;
    out->fmin = fmin;
    out->fmax = fmax;
    out->tsamp = h->tbin;
    out->d_min = static_cast<float>(d_min);
    out->d_max = static_cast<float>(d_max);
    return BFS_OK;
}
