// Coherent-dedispersion chunk stage on sm_100a.
//
// Reference chain (L/CDMT): CSession_guppi_gpu::unpack_chunk
// (Session_guppi_gpu.cu:53-60,117-141) -> CChunk_gpu::process (Chunk_gpu.cu:254-460):
// forward C2C FFT of every nbin-sample segment, then per coherent DM the chirp
// multiply (CChunk_fly_gpu::elementWiseMult, Chunk_fly_gpu.cu:94-163), inverse
// C2C FFTs of length mbin = nbin / len_sft, power detection summed over
// polarisations with a roll by nbin/2 (roll_rows_normalize_sum_kernel,
// Chunk_gpu.cu:476-494), unpadding + frequency reversal into a fine-channel
// plane (transpose_unpadd_intensity, :497-516), a per-row circular
// dedispersion shift (dedisperse, :613-632), statistical preprocessing, the
// FDMT of the mask and of the data, and fdmt_normalization (:327-359).
//
// Layouts (the reference's): raw GUPPI chunk int8 [coarse chan][sample][npol]
// with npol bytes per sample = (re, im) per polarisation; spectra / voltages
// complex64 [pol][fft][coarse chan][nbin]; the FDMT input plane float32
// [fine channel, highest frequency first][msamp].
//
// Differences in form: detection, roll, unpadding, reversal and the
// dedispersion shift are ONE gather kernel here (one read of the voltages,
// one write of the plane) instead of three passes; the chirp phase is FP64
// (modf before sincospi) and the complex multiply FP32 without FMA
// contraction.  For nbin = 2^20 the forward FFT is this library's own, fused
// with the unpack; for mbin = 32768 the chirp, the inverse sub-band
// transforms and the detection are two passes of this library's own
// (subband_ifft: the chirp applied on load from a per-DM table, the detected
// plane written by the second pass); other sizes use cuFFT with the
// reference's sizes.
#include <cufft.h>

#include <cmath>
#include <memory>
#include <vector>

#include "internal.h"

struct bfs_chunk {
    bfs_chunk_desc d;
    int mbin = 0, nov_pc = 0, mbin_adj = 0, msamp = 0, rows = 0;
    int64_t len_chunk = 0;   // samples per coarse channel in one chunk
    int64_t cplx_len = 0;    // complex values of one spectrum / voltage buffer
    cufftHandle fwd = 0, inv = 0;
    bool have_fwd = false, have_inv = false;
    bfs_fdmt_plan* fdmt = nullptr;
    float2* volt = nullptr;  // chirped spectrum, then voltages, per DM
    float* plane = nullptr;  // rows x msamp FDMT input
    float* mask = nullptr;   // rows x msamp normalisation input
    float* norm = nullptr;   // max_dt x msamp FDMT of the mask
    float* buff = nullptr;   // 4 + 2 rows statistics
    int* d_shift = nullptr;  // rows dedispersion shifts
    // chirp factors per coherent DM ([chan][sub-band][mbin]) for the own
    // sub-band transforms, the most recent kChirpCache DMs
    std::vector<std::pair<double, float2*>> chirps;
    ~bfs_chunk() {
        if (have_fwd) cufftDestroy(fwd);
        if (have_inv) cufftDestroy(inv);
        if (fdmt) bfs_fdmt_plan_destroy(fdmt);
        for (auto& c : chirps) cudaFree(c.second);
        for (void* p : {static_cast<void*>(volt), static_cast<void*>(plane), static_cast<void*>(mask),
                        static_cast<void*>(norm), static_cast<void*>(buff), static_cast<void*>(d_shift)})
            if (p) cudaFree(p);
    }
};

namespace bfs {
bool subband_ifft_supported(int nbin, int len_sft, int npol);
bfs_status subband_ifft(const float2* spec, const float2* chirp, float2* z, float* plane, const int* shift,
                        int npol2, int nfft, int nchan, int len_sft, int nbin, int nov_pc, int mbin_adj, int msamp,
                        cudaStream_t s);
bool fft_fused_supported(int nbin, int npol);
bfs_status fft_forward_guppi(const signed char* raw, float2* tmp, float2* x, long long nsamp, int noverlap,
                             int nfft, int nchan, int npol, cudaStream_t s);
namespace {

constexpr double kDispersionConstant = 4.148808e9;  // MHz^2 pc^-1 cm^3 us (Chunk_fly_gpu.cu:139)

// int8 GUPPI -> complex64 with overlap-save zero padding.  One thread per
// (bin, fft, coarse channel); reads all polarisations of a sample at once.
__global__ void k_unpack_guppi(const signed char* __restrict__ raw, float2* __restrict__ out,
                               long long nsamp, int noverlap, int nbin, int nfft, int npol,
                               int nchan) {
    const int ibin = blockIdx.x * blockDim.x + threadIdx.x;
    if (ibin >= nbin) return;
    const int ifft = blockIdx.y, ichan = blockIdx.z;
    const long long isamp = static_cast<long long>(ibin) + static_cast<long long>(nbin - 2 * noverlap) * ifft - noverlap;
    const bool valid = isamp >= 0 && isamp < nsamp;
    const signed char* src = raw + (static_cast<long long>(ichan) * nsamp + (valid ? isamp : 0)) * npol;
    for (int ipol = 0; ipol < npol / 2; ++ipol) {
        const size_t o = (static_cast<size_t>(ipol) * nfft * nchan + static_cast<size_t>(ifft) * nchan + ichan) * nbin + ibin;
        float2 v = make_float2(0.0f, 0.0f);
        if (valid) v = make_float2(static_cast<float>(src[2 * ipol]), static_cast<float>(src[2 * ipol + 1]));
        out[o] = v;
    }
}

// The chirp factor of bin ibin of sub-band isft of coarse channel ichan:
// phase in FP64 (modf before sincospi), taper, 1/nbin, rounded to float.
__device__ __forceinline__ float2 chirp_factor(double dm, int ichan, int isft, int ibin, int len_sft, int mbin,
                                               int nbin, double fmin, double bw_sub, double bw_chan) {
    // centre of the fine channel, rounded to float as the reference stores it
    const float f0 = static_cast<float>(fmin + bw_sub * (0.5 + ichan) +
                                        bw_chan * (isft - len_sft / 2.0 + 0.5));
    const double fb = -0.5 * bw_chan + (ibin + 0.5) * bw_chan / mbin;
    const double taper = 1.0 / sqrt(1.0 + pow(fb / (0.47 * bw_chan), 80));
    const double r = fb / static_cast<double>(f0);
    const double phase = __dmul_rn(__dmul_rn(dm, r), r) / (static_cast<double>(f0) + fb) * kDispersionConstant;
    double whole;
    const double frac = -modf(phase, &whole) * 2.0;
    double sn, cs;
    sincospi(frac, &sn, &cs);
    return make_float2(static_cast<float>(cs * taper / static_cast<double>(nbin)),
                       static_cast<float>(sn * taper / static_cast<double>(nbin)));
}

// Chirp: one thread per (bin of the mbin sub-band, sub-band, coarse channel);
// the factor is applied to every polarisation and FFT segment at the
// fft-shifted position of the nbin spectrum.
__global__ void k_chirp(const float2* __restrict__ in, float2* __restrict__ out, double dm, int nchan,
                        int len_sft, int mbin, int nbin, int nseg, double fmin, double bw_sub,
                        double bw_chan) {
    const int ibin = blockIdx.x * blockDim.x + threadIdx.x;
    if (ibin >= mbin) return;
    const int isft = blockIdx.y, ichan = blockIdx.z;
    const float2 cf = chirp_factor(dm, ichan, isft, ibin, len_sft, mbin, nbin, fmin, bw_sub, bw_chan);
    const size_t pos = static_cast<size_t>(ichan) * nbin + (isft * mbin + ibin + nbin / 2) % nbin;
    const size_t stride = static_cast<size_t>(nbin) * nchan;
    for (int i = 0; i < nseg; ++i) {
        const float2 a = in[pos + i * stride];
        float2 o;
        o.x = __fsub_rn(__fmul_rn(a.x, cf.x), __fmul_rn(a.y, cf.y));
        o.y = __fadd_rn(__fmul_rn(a.x, cf.y), __fmul_rn(a.y, cf.x));
        out[pos + i * stride] = o;
    }
}

// The factors alone: tab[(ichan len_sft + isft) mbin + ibin].
__global__ void k_chirp_table(float2* __restrict__ tab, double dm, int len_sft, int mbin, int nbin, double fmin,
                              double bw_sub, double bw_chan) {
    const int ibin = blockIdx.x * blockDim.x + threadIdx.x;
    if (ibin >= mbin) return;
    const int isft = blockIdx.y, ichan = blockIdx.z;
    tab[(static_cast<size_t>(ichan) * len_sft + isft) * mbin + ibin] =
        chirp_factor(dm, ichan, isft, ibin, len_sft, mbin, nbin, fmin, bw_sub, bw_chan);
}

// Power detection + roll by nbin/2 + unpadding + frequency reversal +
// dedispersion shift, as one gather: output row r (fine channel, highest
// frequency first), columns c .. c + kDetectCols - 1 of the dedispersed plane
// per thread, so that every thread has kDetectCols x npol2 independent
// voltage loads in flight and stores one 16-byte vector when the row allows.
constexpr int kDetectThreads = 256;
constexpr int kDetectCols = 4;

__global__ void __launch_bounds__(kDetectThreads)
k_detect(const float2* __restrict__ volt, float* __restrict__ plane, int nchan, int len_sft, int mbin,
         int nbin, int nfft, int npol2, int nov_pc, int mbin_adj, int msamp, const int* __restrict__ shift,
         double inv_nbin2, int vec_store) {
    const int r = blockIdx.y;
    const int c = (blockIdx.x * kDetectThreads + threadIdx.x) * kDetectCols;
    if (c >= msamp) return;
    // source column of output column c: dedisperse writes out[(idx + s) % msamp] = in[idx]
    int idx = (c - __ldg(shift + r)) % msamp;
    if (idx < 0) idx += msamp;
    const int isub = r / len_sft;
    const int ifine = len_sft - 1 - (r % len_sft);
    const int coarse = nchan - 1 - isub;
    int ifft = idx / mbin_adj;
    int ibin = idx - ifft * mbin_adj;
    int q0 = ifine * mbin + nov_pc + nbin / 2;   // position of ibin 0 before the roll
    if (q0 >= nbin) q0 -= nbin;
    const size_t pol_stride = static_cast<size_t>(nfft) * nchan * nbin;
    float2 v[kDetectCols][2];
#pragma unroll
    for (int j = 0; j < kDetectCols; ++j) {
        int q = q0 + ibin;
        if (q >= nbin) q -= nbin;
        const size_t base = (static_cast<size_t>(ifft) * nchan + coarse) * nbin + q;
        const bool live = c + j < msamp;
#pragma unroll
        for (int ipol = 0; ipol < 2; ++ipol)
            v[j][ipol] = (live && ipol < npol2) ? __ldg(volt + base + ipol * pol_stride) : make_float2(0.f, 0.f);
        // next source column: idx + 1, wrapping at msamp, carried into (ifft, ibin)
        if (++idx == msamp) {
            idx = 0; ifft = 0; ibin = 0;
        } else if (++ibin == mbin_adj) {
            ibin = 0; ++ifft;
        }
    }
    float acc[kDetectCols];
#pragma unroll
    for (int j = 0; j < kDetectCols; ++j) {
        acc[j] = 0.0f;
#pragma unroll
        for (int ipol = 0; ipol < 2; ++ipol) {
            if (ipol >= npol2) break;
            const double x = v[j][ipol].x, y = v[j][ipol].y;
            // |v|^2 / nbin / nbin in FP64 (the reference's roll kernel); with nbin a
            // power of two the two divides are an exact scaling by 2^-2k
            const double pw = inv_nbin2 > 0.0 ? (x * x + y * y) * inv_nbin2 : (x * x + y * y) / nbin / nbin;
            acc[j] = __fadd_rn(acc[j], static_cast<float>(pw));
        }
    }
    float* o = plane + static_cast<size_t>(r) * msamp + c;
    if (vec_store) {   // 16-byte aligned plane, msamp % 4 == 0: every row offset keeps the alignment
        *reinterpret_cast<float4*>(o) = make_float4(acc[0], acc[1], acc[2], acc[3]);
    } else {
#pragma unroll
        for (int j = 0; j < kDetectCols; ++j)
            if (c + j < msamp) o[j] = acc[j];
    }
}

// Complex buffers are read and written as float2: 8-byte alignment.
bool cplx_aligned(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 7) == 0; }

bfs_status cufft_check(cufftResult r, const char* what) {
    if (r == CUFFT_SUCCESS) return BFS_OK;
    return fail(BFS_ERR_CUDA, "%s failed (cufftResult %d)", what, static_cast<int>(r));
}

}  // namespace
}  // namespace bfs

using namespace bfs;

extern "C" int bfs_chunk_coherent_dms(double d_min, double d_max, int ncoherent, double* dms, int cap) {
    // CChunkB::CChunkB (L/CDMT/ChunkB.cpp:171-176): step = d_max / ncoherent,
    // count = (int)((d_max - d_min) / step), dm_i = d_min + i * step
    if (ncoherent <= 0 || !(d_max > 0.0)) return 0;
    const double step = d_max / ncoherent;
    const int n = static_cast<int>((d_max - d_min) / step);
    for (int i = 0; i < n && i < cap; ++i) dms[i] = d_min + i * step;
    return n < 0 ? 0 : n;
}

extern "C" bfs_status bfs_chunk_create(const bfs_chunk_desc* desc, bfs_chunk** out) {
    BFS_ARG(desc && out, "null argument");
    *out = nullptr;
    const bfs_chunk_desc& d = *desc;
    BFS_ARG(d.npol == 2 || d.npol == 4, "npol must be 2 or 4 (got %d)", d.npol);
    BFS_ARG(d.nchan >= 1 && d.len_sft >= 1 && d.nfft >= 1 && d.nbin >= 2, "bad chunk geometry");
    BFS_ARG(d.nbin % d.len_sft == 0, "nbin must be a multiple of len_sft");
    BFS_ARG(d.noverlap >= 0 && 2 * d.noverlap < d.nbin, "bad overlap");
    BFS_ARG(d.tsamp > 0.0f && d.fmax > d.fmin && d.fmin > 0.0f, "bad band or sample time");
    std::unique_ptr<bfs_chunk> c(new bfs_chunk);
    c->d = d;
    // CChunkB geometry (L/CDMT/ChunkB.h:77-98)
    c->mbin = d.nbin / d.len_sft;
    c->nov_pc = d.noverlap / d.len_sft;
    c->mbin_adj = c->mbin - 2 * c->nov_pc;
    BFS_ARG(c->mbin_adj > 0, "overlap leaves no samples per segment");
    c->msamp = d.nfft * c->mbin_adj;
    c->rows = d.nchan * d.len_sft;
    c->len_chunk = static_cast<int64_t>(d.nbin - 2 * d.noverlap) * d.nfft;
    c->cplx_len = static_cast<int64_t>(d.npol / 2) * d.nfft * d.nchan * d.nbin;
    const int max_dt = d.max_dt > 0 ? d.max_dt : d.len_sft;
    c->d.max_dt = max_dt;
    // FFT plans with the reference's sizes (Chunk_gpu.cu:197-209)
    int n = d.nbin;
    {
        bfs_status st = cufft_check(cufftPlanMany(&c->fwd, 1, &n, nullptr, 1, d.nbin, nullptr, 1, d.nbin,
                                                  CUFFT_C2C, d.nfft * d.nchan * d.npol / 2),
                                    "cufftPlanMany(forward)");
        if (st != BFS_OK) return st;
        c->have_fwd = true;
        int m = c->mbin;
        st = cufft_check(cufftPlanMany(&c->inv, 1, &m, nullptr, 1, c->mbin, nullptr, 1, c->mbin,
                                       CUFFT_C2C, d.nfft * d.nchan * d.len_sft * d.npol / 2),
                         "cufftPlanMany(inverse)");
        if (st != BFS_OK) return st;
        c->have_inv = true;
    }
    bfs_fdmt_desc fd{};
    fd.fmin = d.fmin; fd.fmax = d.fmax; fd.nchan = c->rows; fd.ncols = c->msamp; fd.max_dt = max_dt;
    fd.plan_kind = BFS_PLAN_KEITH; fd.precision = BFS_PREC_F32; fd.fuse_depth = -1;
    bfs_status st = bfs_fdmt_plan_create(&fd, &c->fdmt);
    if (st != BFS_OK) return st;
    BFS_CUDA(cudaMalloc(&c->volt, sizeof(float2) * c->cplx_len));
    BFS_CUDA(cudaMalloc(&c->plane, sizeof(float) * static_cast<size_t>(c->rows) * c->msamp));
    BFS_CUDA(cudaMalloc(&c->mask, sizeof(float) * static_cast<size_t>(c->rows) * c->msamp));
    BFS_CUDA(cudaMalloc(&c->norm, sizeof(float) * static_cast<size_t>(max_dt) * c->msamp));
    BFS_CUDA(cudaMalloc(&c->buff, sizeof(float) * (4 + 2 * static_cast<size_t>(c->rows))));
    BFS_CUDA(cudaMalloc(&c->d_shift, sizeof(int) * c->rows));
    *out = c.release();
    return BFS_OK;
}

extern "C" bfs_status bfs_chunk_destroy(bfs_chunk* c) {
    delete c;
    return BFS_OK;
}

extern "C" bfs_status bfs_chunk_info(const bfs_chunk* c, int64_t* info, int cap) {
    BFS_ARG(c && info && cap >= 8, "need 8 entries");
    info[0] = c->mbin; info[1] = c->nov_pc; info[2] = c->mbin_adj; info[3] = c->msamp;
    info[4] = c->rows; info[5] = c->len_chunk; info[6] = c->cplx_len; info[7] = c->d.max_dt;
    return BFS_OK;
}

extern "C" bfs_status bfs_chunk_unpack(bfs_chunk* c, const int8_t* d_raw, void* d_cplx, void* stream) {
    BFS_ARG(c && d_raw && d_cplx, "null argument");
    BFS_ARG(cplx_aligned(d_cplx), "d_cplx must be 8-byte aligned");
    const bfs_chunk_desc& d = c->d;
    dim3 grid((d.nbin + 255) / 256, d.nfft, d.nchan);
    BFS_ARG(grid.y <= 65535 && grid.z <= 65535, "too many segments or channels");
    k_unpack_guppi<<<grid, 256, 0, as_stream(stream)>>>(reinterpret_cast<const signed char*>(d_raw),
                                                         static_cast<float2*>(d_cplx), c->len_chunk,
                                                         d.noverlap, d.nbin, d.nfft, d.npol, d.nchan);
    BFS_LAUNCH_CHECK("k_unpack_guppi");
    return BFS_OK;
}

extern "C" bfs_status bfs_chunk_forward_fft(bfs_chunk* c, void* d_cplx, void* stream) {
    BFS_ARG(c && d_cplx, "null argument");
    BFS_ARG(cplx_aligned(d_cplx), "d_cplx must be 8-byte aligned");
    bfs_status st = cufft_check(cufftSetStream(c->fwd, as_stream(stream)), "cufftSetStream");
    if (st != BFS_OK) return st;
    return cufft_check(cufftExecC2C(c->fwd, static_cast<cufftComplex*>(d_cplx),
                                    static_cast<cufftComplex*>(d_cplx), CUFFT_FORWARD),
                       "cufftExecC2C(forward)");
}

constexpr size_t kChirpCache = 4;

// Whether the DM loop runs the own sub-band transforms (chirp table + two
// passes) for these buffers.
static bool own_subband(const bfs_chunk* c, const void* d_spec) {
    return subband_ifft_supported(c->d.nbin, c->d.len_sft, c->d.npol) &&
           reinterpret_cast<uintptr_t>(d_spec) % 16 == 0;
}

// The chirp table of one coherent DM (computed on first use, kept for the
// chunk's most recent DMs).
static bfs_status chirp_table(bfs_chunk* c, double dm, const float2** out, cudaStream_t s) {
    for (auto& e : c->chirps)
        if (e.first == dm) { *out = e.second; return BFS_OK; }
    const bfs_chunk_desc& d = c->d;
    float2* tab = nullptr;
    if (c->chirps.size() >= kChirpCache) {   // reuse the oldest table's memory
        BFS_CUDA(cudaStreamSynchronize(s));
        tab = c->chirps.front().second;
        c->chirps.erase(c->chirps.begin());
    } else {
        BFS_CUDA(cudaMalloc(&tab, sizeof(float2) * static_cast<size_t>(d.nchan) * d.len_sft * c->mbin));
    }
    c->chirps.emplace_back(dm, tab);
    const double bw = static_cast<double>(d.fmax - d.fmin);
    const double bw_sub = bw / d.nchan;
    const double bw_chan = bw_sub / d.len_sft;
    dim3 grid((c->mbin + 255) / 256, d.len_sft, d.nchan);
    BFS_ARG(grid.y <= 65535 && grid.z <= 65535, "too many sub-bands or channels");
    k_chirp_table<<<grid, 256, 0, s>>>(tab, dm, d.len_sft, c->mbin, d.nbin, static_cast<double>(d.fmin), bw_sub,
                                       bw_chan);
    BFS_LAUNCH_CHECK("k_chirp_table");
    *out = tab;
    return BFS_OK;
}

static bfs_status chunk_voltages(bfs_chunk* c, const void* d_spec, double dm, float2* d_volt,
                                 cudaStream_t s) {
    const bfs_chunk_desc& d = c->d;
    // (the first pass reads all of a sub-band while writing it: not in place)
    const char* sp = static_cast<const char*>(d_spec);
    const char* vp = reinterpret_cast<const char*>(d_volt);
    const size_t bytes = sizeof(float2) * static_cast<size_t>(c->cplx_len);
    const bool apart = vp + bytes <= sp || sp + bytes <= vp;
    if (apart && own_subband(c, d_spec)) {
        const float2* tab = nullptr;
        bfs_status st = chirp_table(c, dm, &tab, s);
        if (st != BFS_OK) return st;
        return subband_ifft(static_cast<const float2*>(d_spec), tab, d_volt, nullptr, nullptr, d.npol / 2, d.nfft,
                            d.nchan, d.len_sft, d.nbin, c->nov_pc, c->mbin_adj, c->msamp, s);
    }
    // band arithmetic as in CChunk_fly_gpu::elementWiseMult (Chunk_fly_gpu.cu:96-99)
    const double bw = static_cast<double>(d.fmax - d.fmin);
    const double bw_sub = bw / d.nchan;
    const double bw_chan = bw_sub / d.len_sft;
    dim3 grid((c->mbin + 255) / 256, d.len_sft, d.nchan);
    BFS_ARG(grid.y <= 65535 && grid.z <= 65535, "too many sub-bands or channels");
    k_chirp<<<grid, 256, 0, s>>>(static_cast<const float2*>(d_spec), d_volt, dm, d.nchan, d.len_sft,
                                 c->mbin, d.nbin, d.nfft * d.npol / 2, static_cast<double>(d.fmin),
                                 bw_sub, bw_chan);
    BFS_LAUNCH_CHECK("k_chirp");
    bfs_status st = cufft_check(cufftSetStream(c->inv, s), "cufftSetStream");
    if (st != BFS_OK) return st;
    return cufft_check(cufftExecC2C(c->inv, reinterpret_cast<cufftComplex*>(d_volt),
                                    reinterpret_cast<cufftComplex*>(d_volt), CUFFT_INVERSE),
                       "cufftExecC2C(inverse)");
}

extern "C" bfs_status bfs_chunk_voltages(bfs_chunk* c, const void* d_spec, double dm, void* d_volt,
                                         void* stream) {
    BFS_ARG(c && d_spec && d_volt, "null argument");
    BFS_ARG(cplx_aligned(d_spec) && cplx_aligned(d_volt), "d_spec and d_volt must be 8-byte aligned");
    return chunk_voltages(c, d_spec, dm, static_cast<float2*>(d_volt), as_stream(stream));
}

// Dedispersion shifts of the fine-channel rows (dedisperse, Chunk_gpu.cu:613-632):
// row i has frequency fmin + (rows-1-i) * foff and moves by
// round(4148.808 * dm * (fmin^-2 - f^-2) / (len_sft * tsamp)).
static void chunk_shifts(const bfs_chunk* c, double dm, std::vector<int>& sh) {
    const bfs_chunk_desc& d = c->d;
    const double fmin = d.fmin;
    const double foff = (static_cast<double>(d.fmax) - static_cast<double>(d.fmin)) / (d.nchan * d.len_sft);
    const double tw = static_cast<double>(static_cast<float>(d.len_sft) * d.tsamp);
    sh.resize(c->rows);
    for (int i = 0; i < c->rows; ++i) {
        const double f = static_cast<double>(c->rows - 1 - i) * foff + fmin;
        const double delay = 4.148808e3 * dm * (1.0 / (fmin * fmin) - 1.0 / (f * f));
        sh[i] = static_cast<int>(std::round(delay / tw));
    }
}

static bfs_status chunk_detect(bfs_chunk* c, const float2* d_volt, double dm, float* d_plane,
                               cudaStream_t s) {
    std::vector<int> sh;
    chunk_shifts(c, dm, sh);
    BFS_CUDA(cudaMemcpyAsync(c->d_shift, sh.data(), sizeof(int) * sh.size(), cudaMemcpyHostToDevice, s));
    const bfs_chunk_desc& d = c->d;
    const int span = kDetectThreads * kDetectCols;
    dim3 grid((c->msamp + span - 1) / span, c->rows);
    BFS_ARG(grid.y <= 65535, "too many fine channels");
    BFS_ARG(d.npol / 2 <= 2, "at most two polarisations");
    const bool pow2 = (d.nbin & (d.nbin - 1)) == 0;
    const double inv_nbin2 = pow2 ? 1.0 / (static_cast<double>(d.nbin) * d.nbin) : 0.0;  // exact for 2^k
    const int vec_store = (c->msamp % 4 == 0) && (reinterpret_cast<uintptr_t>(d_plane) & 15) == 0;
    k_detect<<<grid, kDetectThreads, 0, s>>>(d_volt, d_plane, d.nchan, d.len_sft, c->mbin, d.nbin, d.nfft,
                                  d.npol / 2, c->nov_pc, c->mbin_adj, c->msamp, c->d_shift, inv_nbin2,
                                  vec_store);
    BFS_LAUNCH_CHECK("k_detect");
    // the host vector must outlive the (pageable, staged) copy: wait for it
    BFS_CUDA(cudaStreamSynchronize(s));
    return BFS_OK;
}

// The detected plane of one DM straight from the spectrum: the own two-pass
// chirp + sub-band transforms + detection when the geometry has them (the
// voltages never stored), else voltages into c->volt and the gather.
static bfs_status chunk_detect_spectrum(bfs_chunk* c, const void* d_spec, double dm, float* d_plane,
                                        cudaStream_t s) {
    if (!own_subband(c, d_spec)) {
        bfs_status st = chunk_voltages(c, d_spec, dm, c->volt, s);
        if (st != BFS_OK) return st;
        return chunk_detect(c, c->volt, dm, d_plane, s);
    }
    std::vector<int> sh;
    chunk_shifts(c, dm, sh);
    BFS_CUDA(cudaMemcpyAsync(c->d_shift, sh.data(), sizeof(int) * sh.size(), cudaMemcpyHostToDevice, s));
    const float2* tab = nullptr;
    bfs_status st = chirp_table(c, dm, &tab, s);
    if (st == BFS_OK) {
        const bfs_chunk_desc& d = c->d;
        st = subband_ifft(static_cast<const float2*>(d_spec), tab, c->volt, d_plane, c->d_shift, d.npol / 2, d.nfft,
                          d.nchan, d.len_sft, d.nbin, c->nov_pc, c->mbin_adj, c->msamp, s);
    }
    // the host vector must outlive the (pageable, staged) copy
    cudaError_t e = cudaStreamSynchronize(s);
    if (st == BFS_OK && e != cudaSuccess) st = fail(BFS_ERR_CUDA, "cudaStreamSynchronize: %s", cudaGetErrorString(e));
    return st;
}

extern "C" bfs_status bfs_chunk_detect_spectrum(bfs_chunk* c, const void* d_spec, double dm, float* d_plane,
                                                void* stream) {
    BFS_ARG(c && d_spec && d_plane, "null argument");
    BFS_ARG(cplx_aligned(d_spec), "d_spec must be 8-byte aligned");
    return chunk_detect_spectrum(c, d_spec, dm, d_plane, as_stream(stream));
}

extern "C" bfs_status bfs_chunk_detect(bfs_chunk* c, const void* d_volt, double dm, float* d_plane,
                                       void* stream) {
    BFS_ARG(c && d_volt && d_plane, "null argument");
    BFS_ARG(cplx_aligned(d_volt), "d_volt must be 8-byte aligned");
    return chunk_detect(c, static_cast<const float2*>(d_volt), dm, d_plane, as_stream(stream));
}

extern "C" bfs_status bfs_chunk_unpack_fft(bfs_chunk* c, const int8_t* d_raw, void* d_spec, void* stream) {
    BFS_ARG(c && d_raw && d_spec, "null argument");
    BFS_ARG(cplx_aligned(d_spec), "d_spec must be 8-byte aligned");
    const bfs_chunk_desc& d = c->d;
    // the fused transform reads whole samples (npol bytes) as one word and
    // writes float2s: it needs the raw chunk npol-aligned and d_spec 8-aligned
    const bool aligned = (reinterpret_cast<uintptr_t>(d_raw) % d.npol) == 0 &&
                         (reinterpret_cast<uintptr_t>(d_spec) % sizeof(float2)) == 0;
    if (aligned && fft_fused_supported(d.nbin, d.npol))
        return fft_forward_guppi(reinterpret_cast<const signed char*>(d_raw), c->volt, static_cast<float2*>(d_spec),
                                 c->len_chunk, d.noverlap, d.nfft, d.nchan, d.npol, as_stream(stream));
    bfs_status st = bfs_chunk_unpack(c, d_raw, d_spec, stream);
    if (st != BFS_OK) return st;
    return bfs_chunk_forward_fft(c, d_spec, stream);
}

// Per coherent DM: voltages, detection, preprocessing, FDMT of mask and data,
// fdmt_normalization (the loop of CChunk_gpu::process after its forward FFT).
static bfs_status chunk_dm_loop(bfs_chunk* c, const void* d_cplx, const double* dms, int ndm, float* d_out,
                                void* stream) {
    cudaStream_t s = as_stream(stream);
    bfs_status st = BFS_OK;
    const size_t plane_out = static_cast<size_t>(c->d.max_dt) * c->msamp;
    for (int i = 0; i < ndm; ++i) {
        st = chunk_detect_spectrum(c, d_cplx, dms[i], c->plane, s);
        if (st != BFS_OK) return st;
        st = bfs_preproc_calc_fdmt_inputs(c->plane, c->rows, c->msamp, c->buff, c->mask, stream);
        if (st != BFS_OK) return st;
        // FDMT of the mask: its rows are all 0 or all 1 (calc_fdmt_inputs zaps
        // whole rows), so the channel-count form gives the same bits in one pass
        st = bfs_fdmt_execute_row_mask(c->fdmt, c->mask, c->msamp, c->norm, stream);
        if (st != BFS_OK) return st;
        float* out = d_out + i * plane_out;
        st = bfs_fdmt_execute(c->fdmt, c->plane, out, 0, stream);
        if (st != BFS_OK) return st;
        st = bfs_fdmt_normalize(out, c->norm, static_cast<int64_t>(plane_out), out, stream);
        if (st != BFS_OK) return st;
    }
    return BFS_OK;
}

extern "C" bfs_status bfs_chunk_process(bfs_chunk* c, void* d_cplx, const double* dms, int ndm,
                                        float* d_out, void* stream) {
    BFS_ARG(c && d_cplx && d_out && (ndm == 0 || dms), "null argument");
    BFS_ARG(cplx_aligned(d_cplx), "d_cplx must be 8-byte aligned");
    bfs_status st = bfs_chunk_forward_fft(c, d_cplx, stream);
    if (st != BFS_OK) return st;
    return chunk_dm_loop(c, d_cplx, dms, ndm, d_out, stream);
}

extern "C" bfs_status bfs_chunk_process_spectrum(bfs_chunk* c, const void* d_spec, const double* dms, int ndm,
                                                 float* d_out, void* stream) {
    BFS_ARG(c && d_spec && d_out && (ndm == 0 || dms), "null argument");
    BFS_ARG(cplx_aligned(d_spec), "d_spec must be 8-byte aligned");
    return chunk_dm_loop(c, d_spec, dms, ndm, d_out, stream);
}

extern "C" bfs_status bfs_chunk_process_raw(bfs_chunk* c, const int8_t* d_raw, void* d_spec, const double* dms,
                                            int ndm, float* d_out, void* stream) {
    BFS_ARG(c && d_raw && d_spec && d_out && (ndm == 0 || dms), "null argument");
    BFS_ARG(cplx_aligned(d_spec), "d_spec must be 8-byte aligned");
    bfs_status st = bfs_chunk_unpack_fft(c, d_raw, d_spec, stream);
    if (st != BFS_OK) return st;
    return chunk_dm_loop(c, d_spec, dms, ndm, d_out, stream);
}
