// Forward FFT of the 2^20-sample coherent-dedispersion segments, fused with
// the GUPPI unpack (sm_100a).
//
// The reference unpacks the int8 chunk into a complex buffer
// (unpack_chunk_guppi_gpu, L/CDMT/Session_guppi_gpu.cu:117-141) and then runs
// cuFFT's C2C forward transform of length nbin on every (pol, fft, channel)
// segment (CChunk_gpu::process, L/CDMT/Chunk_gpu.cu:267).  Here, for
// nbin = 2^20, the two steps are two kernels of a four-step transform
// (N = N1 N2, N1 = N2 = 1024; n = n1 N2 + n2, k = k2 N1 + k1):
//   column pass  B[k1][n2] = W_N^(n2 k1) sum_n1 x[n1 N2 + n2] W_N1^(n1 k1), with
//                x read straight from the int8 samples (overlap-save zeros
//                included), both polarisations of a sample in one 4-byte load;
//   row pass     X[k2 N1 + k1] = sum_n2 B[k1][n2] W_N2^(n2 k2), written in
//                natural order.
// Each 1024-point transform is one warp: 32 points per lane, a 32-point
// radix-2 transform in registers, a twiddle W_1024^(b m1), an exchange through
// a padded 32 x 33 shared tile, and a second 32-point transform.  Twiddles
// come from small tables rounded once from FP64 (products of two table values
// where a full table would not fit on chip).  The result agrees with the unpack + cuFFT
// form to FP32 rounding (it is not bit-identical: a different FFT).
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <vector>

#include "internal.h"

namespace bfs {
namespace {

constexpr int kF = 1024;          // both factors of the four-step transform
constexpr long long kFftN = static_cast<long long>(kF) * kF;
constexpr int kTile = 33;         // padded row of a warp's 32 x 32 exchange tile
constexpr int kRegion = 32 * kTile + 4;  // float2 per warp region (the +4 staggers regions' banks)
constexpr int kColCols = 4;       // columns per CTA in the column pass
constexpr int kRowRows = 4;       // rows per CTA in the row pass (32-byte output runs)
constexpr int kSubN = 32 * kF;    // sub-band transforms of the coherent stage (mbin = 32768)

// cos(pi k / 16), k = 0..8, each rounded once to float (sin(pi k/16) = cos16(8-k)).
__host__ __device__ constexpr float cos16(int k) {
    return k == 0 ? 1.0f : k == 1 ? 0x1.f6297cp-1f : k == 2 ? 0x1.d906bcp-1f : k == 3 ? 0x1.a9b662p-1f
         : k == 4 ? 0x1.6a09e6p-1f : k == 5 ? 0x1.1c73b4p-1f : k == 6 ? 0x1.87de2ap-2f
         : k == 7 ? 0x1.8f8b84p-3f : 0.0f;
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// d * W_32^k, W_32 = exp(-2 pi i / 32), k = 0..15 a compile-time constant
// after unrolling (k = 0 and 8 exact).
__device__ __forceinline__ float2 tw32(float2 d, int k) {
    if (k == 0) return d;
    if (k == 8) return make_float2(d.y, -d.x);
    const float2 w = k < 8 ? make_float2(cos16(k), -cos16(8 - k)) : make_float2(-cos16(16 - k), -cos16(k - 8));
    return cmul(d, w);
}

__host__ __device__ constexpr int bitrev5(int k) {
    return ((k & 1) << 4) | ((k & 2) << 2) | (k & 4) | ((k & 8) >> 2) | ((k & 16) >> 4);
}

// In-place 32-point forward DFT of r (decimation in frequency): afterwards
// X[k] = r[bitrev5(k)].
__device__ __forceinline__ void dft32(float2 (&r)[32]) {
#pragma unroll
    for (int h = 16; h >= 1; h >>= 1) {
#pragma unroll
        for (int g = 0; g < 32; g += 2 * h) {
#pragma unroll
            for (int j = 0; j < h; ++j) {
                const float2 a = r[g + j], b = r[g + j + h];
                r[g + j] = make_float2(a.x + b.x, a.y + b.y);
                r[g + j + h] = tw32(make_float2(a.x - b.x, a.y - b.y), j * (16 / h));
            }
        }
    }
}

// 1024-point forward DFT of one warp.  On entry lane b holds v[32 a + b] in
// r[a]; tile is the warp's 32 x kTile exchange area, tw the shared table
// {W_32^q (q < 32), W_1024^r (r < 32)}: W_1024^(b m1) = W_32^(b m1 / 32)
// W_1024^(b m1 mod 32).  On exit lane m1 holds V[m1 + 32 m2] in r[bitrev5(m2)].
__device__ __forceinline__ void fft1024_warp(float2 (&r)[32], float2* __restrict__ tile,
                                             const float2* __restrict__ tw) {
    const int lane = threadIdx.x & 31;
    dft32(r);  // over a: U_b[m1] = r[bitrev5(m1)]
#pragma unroll
    for (int m1 = 0; m1 < 32; ++m1) {
        const int e = lane * m1;
        tile[lane * kTile + m1] = cmul(r[bitrev5(m1)], cmul(tw[e >> 5], tw[32 + (e & 31)]));
    }
    __syncwarp();
#pragma unroll
    for (int b = 0; b < 32; ++b) r[b] = tile[b * kTile + lane];
    __syncwarp();
    dft32(r);  // over b
}

// Column pass.  grid (kF / kColCols, nfft, nchan); NP2 polarisations.  Warp w
// transforms column c0 + (w % kColCols) of polarisation w / kColCols.
template <int NP2>
__global__ void __launch_bounds__(32 * NP2 * kColCols)
k_fft_cols_guppi(const signed char* __restrict__ raw, float2* __restrict__ y, const float2* __restrict__ tw_g,
                 const float2* __restrict__ twa, const float2* __restrict__ twb, long long nsamp, int noverlap,
                 int nfft, int nchan) {
    constexpr int kWarps = NP2 * kColCols;
    constexpr int kThreads = 32 * kWarps;
    constexpr int kPer = kF * kColCols / kThreads;  // staged samples per thread
    extern __shared__ float2 sm_cols[];
    float2* tw = sm_cols;                       // W_32^q, W_1024^r
    float2* reg = sm_cols + 64;                 // kWarps regions
    const int c0 = blockIdx.x * kColCols;
    const int ifft = blockIdx.y, ichan = blockIdx.z;
    if (threadIdx.x < 64) tw[threadIdx.x] = __ldg(tw_g + threadIdx.x);
    // stage the int8 samples of the CTA's columns: element (n1, c), c fastest,
    // every load of a thread in flight before the first store
    const long long shift = static_cast<long long>(kFftN - 2 * noverlap) * ifft - noverlap;
    const signed char* base = raw + static_cast<long long>(ichan) * nsamp * (2 * NP2);
    int q[kPer];
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        const int e = threadIdx.x + k * kThreads;
        const int c = e % kColCols, n1 = e / kColCols;
        const long long isamp = static_cast<long long>(n1) * kF + c0 + c + shift;
        q[k] = 0;
        if (isamp >= 0 && isamp < nsamp) {
            if (NP2 == 2) q[k] = __ldg(reinterpret_cast<const int*>(base + isamp * 4));
            else q[k] = __ldg(reinterpret_cast<const short*>(base + isamp * 2));
        }
    }
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        const int e = threadIdx.x + k * kThreads;
        const int c = e % kColCols, n1 = e / kColCols;
        const char4 b = *reinterpret_cast<const char4*>(&q[k]);  // bytes re0, im0, re1, im1
        reg[c * kRegion + n1] = make_float2(b.x, b.y);
        if (NP2 == 2) reg[(kColCols + c) * kRegion + n1] = make_float2(b.z, b.w);
    }
    __syncthreads();
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float2* tile = reg + w * kRegion;
    float2 r[32];
#pragma unroll
    for (int a = 0; a < 32; ++a) r[a] = tile[32 * a + lane];
    __syncwarp();
    fft1024_warp(r, tile, tw);
    // the column's k1 = m1 + 32 m2, times W_N^(n2 k1) = W_N^(n2 m1) W_N^(32 n2 m2):
    // one value per lane and one per m2, the same for the whole warp
    const int n2 = c0 + (w % kColCols);
    const float2 wa = __ldg(twa + n2 * 32 + lane);
    const float2* wb = twb + n2 * 32;
    __syncwarp();
#pragma unroll
    for (int m2 = 0; m2 < 32; ++m2) tile[lane + 32 * m2] = cmul(r[bitrev5(m2)], cmul(wa, __ldg(wb + m2)));
    __syncthreads();
    // store rows k1 of every column: y[seg][k1][c0 .. c0 + kColCols)
    const size_t seg0 = static_cast<size_t>(ifft) * nchan + ichan;
    const size_t pol_stride = static_cast<size_t>(nfft) * nchan * kFftN;
#pragma unroll 4
    for (int e = threadIdx.x; e < kF * kWarps; e += kThreads) {
        const int c = e % kColCols, p = (e / kColCols) % NP2, k1 = e / (kColCols * NP2);
        y[p * pol_stride + seg0 * kFftN + static_cast<size_t>(k1) * kF + c0 + c] = reg[(p * kColCols + c) * kRegion + k1];
    }
}

// Row pass.  grid (kF / kRowRows, segments); warp w transforms row
// r0 + w (contiguous over n2) and the CTA writes X[k2 N1 + r0 .. + kRowRows).
__global__ void __launch_bounds__(32 * kRowRows)
k_fft_rows(const float2* __restrict__ y, float2* __restrict__ x, const float2* __restrict__ tw_g) {
    extern __shared__ float2 sm_rows[];
    float2* tw = sm_rows;
    float2* reg = sm_rows + 64;
    const int r0 = blockIdx.x * kRowRows;
    const size_t seg = blockIdx.y;
    if (threadIdx.x < 64) tw[threadIdx.x] = __ldg(tw_g + threadIdx.x);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const float2* row = y + seg * kFftN + static_cast<size_t>(r0 + w) * kF;
    float2 r[32];
#pragma unroll
    for (int a = 0; a < 32; ++a) r[a] = __ldg(row + 32 * a + lane);
    __syncthreads();  // twiddle table staged
    float2* tile = reg + w * kRegion;
    fft1024_warp(r, tile, tw);
    __syncwarp();
#pragma unroll
    for (int m2 = 0; m2 < 32; ++m2) tile[lane + 32 * m2] = r[bitrev5(m2)];
    __syncthreads();
    float2* out = x + seg * kFftN + r0;
#pragma unroll 4
    for (int e = threadIdx.x; e < kF * kRowRows; e += 32 * kRowRows) {
        const int rr = e % kRowRows, k2 = e / kRowRows;
        out[static_cast<size_t>(k2) * kF + rr] = reg[rr * kRegion + k2];
    }
}

// ---- inverse sub-band transforms of the coherent stage ------------------------
// Every mbin = 32768-sample sub-band of the chirped spectrum is transformed
// back (CChunk_fly_gpu::elementWiseMult + the inverse cufftExecC2C of
// CChunk_gpu::process, L/CDMT/Chunk_fly_gpu.cu:94-163, Chunk_gpu.cu:288-290).
// v = IDFT(x) is computed as conj(DFT(conj(x))), the forward DFT of
// y = conj(chirp x) by four steps with m = 32 a + b (a < 1024, b < 32) and
// n = c + 1024 d (c < 1024, d < 32):
//   pass A  Z[b][c] = W_N^(b c) sum_a y[32 a + b] W_1024^(a c)   (one warp per b)
//   pass B  Y[c + 1024 d] = sum_b Z[b][c] W_32^(b d)               (one thread per c)
// and v = conj(Y).  The chirp is read from a per-DM table of the factors
// k_chirp applies (the same FP32 products), so the FP64 phase is evaluated
// once per (channel, sub-band, bin), not once per polarisation and FFT
// segment.  Pass A stores Z in the sub-band's own place (Z[b][c] at offset
// 1024 b + c), pass B either writes v over it (each thread reads and writes
// the same 32 offsets) or detects: |v|^2 / nbin^2 summed over the
// polarisations, rolled, unpadded, reversed and shifted as k_detect does,
// straight into the dedispersed plane.
constexpr int kSubCols = 8;              // pass A: columns b per CTA
constexpr int kSubStage = kF + 1;        // staged column length (the +1 staggers the columns' banks)
constexpr int kSubArea = (kSubCols * kSubStage > kSubCols * kRegion) ? kSubCols * kSubStage : kSubCols * kRegion;
constexpr size_t kSubColSmem = sizeof(float2) * (64 + static_cast<size_t>(kSubArea));
constexpr int kSubRowThreads = 128;      // pass B: values of c per CTA

// Pass A.  blockIdx.x = seg + nseg (cb + 4 sub): the segments of one
// (sub-band, column block) are neighbours, so they share the chirp table's
// block through L2.  spec / chirp 16-byte aligned (two complex per load).
__global__ void __launch_bounds__(32 * kSubCols)
k_subfft_cols(const float2* __restrict__ spec, const float2* __restrict__ chirp, float2* __restrict__ z,
              const float2* __restrict__ tw_g, const float2* __restrict__ sa, const float2* __restrict__ sb,
              int nseg, int nchan, int len_sft, int nbin) {
    constexpr int kThreads = 32 * kSubCols;
    constexpr int kBlk = 32 / kSubCols;
    constexpr int kQ = kF * kSubCols / 2;   // float4s (two complex) per CTA
    constexpr int kBatch = 8;               // float4 loads of each array in flight per thread
    extern __shared__ float2 sm_sub[];
    float2* tw = sm_sub;
    float2* area = sm_sub + 64;
    int id = blockIdx.x;
    const int seg = id % nseg;
    id /= nseg;
    const int cb = id % kBlk, sub = id / kBlk;
    const int ichan = sub / len_sft, isft = sub % len_sft;
    const int b0 = cb * kSubCols;
    const int chunk = (isft + len_sft / 2) % len_sft;   // fft-shifted place of the sub-band
    const size_t base = (static_cast<size_t>(seg) * nchan + ichan) * nbin + static_cast<size_t>(chunk) * kSubN;
    const float4* x4 = reinterpret_cast<const float4*>(spec + base);
    const float4* c4 = reinterpret_cast<const float4*>(chirp + static_cast<size_t>(sub) * kSubN);
    if (threadIdx.x < 64) tw[threadIdx.x] = __ldg(tw_g + threadIdx.x);
#pragma unroll
    for (int k0 = 0; k0 < kQ / kThreads; k0 += kBatch) {
        float4 q[kBatch], c[kBatch];
#pragma unroll
        for (int k = 0; k < kBatch; ++k) {
            const int e = threadIdx.x + (k0 + k) * kThreads;   // (a, pair jj) = (e / 4, e % 4)
            const int off = (32 * (e >> 2) + b0 + 2 * (e & 3)) >> 1;
            q[k] = __ldg(x4 + off);
            c[k] = __ldg(c4 + off);
        }
#pragma unroll
        for (int k = 0; k < kBatch; ++k) {
            const int e = threadIdx.x + (k0 + k) * kThreads;
            const int a = e >> 2, jj = 2 * (e & 3);
            // y = conj(x * chirp), the product as k_chirp forms it
            const float ox0 = __fsub_rn(__fmul_rn(q[k].x, c[k].x), __fmul_rn(q[k].y, c[k].y));
            const float oy0 = __fadd_rn(__fmul_rn(q[k].x, c[k].y), __fmul_rn(q[k].y, c[k].x));
            const float ox1 = __fsub_rn(__fmul_rn(q[k].z, c[k].z), __fmul_rn(q[k].w, c[k].w));
            const float oy1 = __fadd_rn(__fmul_rn(q[k].z, c[k].w), __fmul_rn(q[k].w, c[k].z));
            area[jj * kSubStage + a] = make_float2(ox0, -oy0);
            area[(jj + 1) * kSubStage + a] = make_float2(ox1, -oy1);
        }
    }
    __syncthreads();
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float2 r[32];
#pragma unroll
    for (int a = 0; a < 32; ++a) r[a] = area[w * kSubStage + 32 * a + lane];
    __syncthreads();   // every column is in registers: the area becomes the exchange tiles
    fft1024_warp(r, area + w * kRegion, tw);
    // Z[b][m1 + 32 m2] = V[m1 + 32 m2] W_N^(b m1) W_1024^(b m2)
    const int b = b0 + w;
    const float2 wa = __ldg(sa + b * 32 + lane);
    float2* zb = z + base + static_cast<size_t>(b) * kF;
#pragma unroll
    for (int m2 = 0; m2 < 32; ++m2) zb[lane + 32 * m2] = cmul(r[bitrev5(m2)], cmul(wa, __ldg(sb + b * 32 + m2)));
}

// Pass B.  blockIdx.x = cb + 8 id with id = (fft, coarse channel, sub-band)
// (DETECT: both polarisations) or (segment, coarse channel, sub-band).
template <bool DETECT>
__global__ void __launch_bounds__(kSubRowThreads)
k_subfft_rows(float2* __restrict__ z, float* __restrict__ plane, const int* __restrict__ shift, int npol2,
              int nfft, int nchan, int len_sft, int nbin, int nov_pc, int mbin_adj, int msamp, double inv_nbin2) {
    constexpr int kBlk = kF / kSubRowThreads;
    int id = blockIdx.x;
    const int c = (id % kBlk) * kSubRowThreads + threadIdx.x;
    id /= kBlk;
    const int isft = id % len_sft;
    id /= len_sft;
    const int ichan = id % nchan, outer = id / nchan;   // outer: fft (DETECT) or segment
    const size_t sub_off = static_cast<size_t>((isft + len_sft / 2) % len_sft) * kSubN + c;
    float2 r[32];
    if constexpr (!DETECT) {
        float2* zz = z + (static_cast<size_t>(outer) * nchan + ichan) * nbin + sub_off;
#pragma unroll
        for (int b = 0; b < 32; ++b) r[b] = zz[static_cast<size_t>(b) * kF];
        dft32(r);
#pragma unroll
        for (int d = 0; d < 32; ++d) {
            const float2 y = r[bitrev5(d)];
            zz[static_cast<size_t>(d) * kF] = make_float2(y.x, -y.y);
        }
    } else {
    float acc[32];
#pragma unroll
    for (int d = 0; d < 32; ++d) acc[d] = 0.0f;
    for (int p = 0; p < npol2; ++p) {
        const float2* zz = z + ((static_cast<size_t>(p) * nfft + outer) * nchan + ichan) * nbin + sub_off;
#pragma unroll
        for (int b = 0; b < 32; ++b) r[b] = __ldg(zz + static_cast<size_t>(b) * kF);
        dft32(r);
#pragma unroll
        for (int d = 0; d < 32; ++d) {
            // |v|^2 / nbin / nbin in FP64 (x^2 and y^2 of floats are exact in
            // double; nbin a power of two: the scaling is exact), then FP32
            const float2 y = r[bitrev5(d)];
            const double px = y.x, py = y.y;
            acc[d] = __fadd_rn(acc[d], static_cast<float>((px * px + py * py) * inv_nbin2));
        }
    }
    const int row = (nchan - 1 - ichan) * len_sft + (len_sft - 1 - isft);
    const int sh = __ldg(shift + row);
    float* out = plane + static_cast<size_t>(row) * msamp;
#pragma unroll
    for (int d = 0; d < 32; ++d) {
        const int n = c + kF * d;
        if (n >= nov_pc && n < nov_pc + mbin_adj) {
            const long long idx = static_cast<long long>(outer) * mbin_adj + (n - nov_pc);
            long long col = (idx + sh) % msamp;
            if (col < 0) col += msamp;
            out[col] = acc[d];
        }
    }
    }
}

constexpr size_t kColSmem(int np2) { return sizeof(float2) * (64 + static_cast<size_t>(np2) * kColCols * kRegion); }
constexpr size_t kRowSmem = sizeof(float2) * (64 + static_cast<size_t>(kRowRows) * kRegion);

// Twiddle tables of one device, each value rounded once from FP64:
// small = {W_32^q, q < 32; W_1024^r, r < 32}; twa[n2][m1] = W_N^(n2 m1),
// twb[n2][m2] = W_N^(32 n2 m2) (n2 < 1024; m1, m2 < 32).
struct FftTables {
    float2* small = nullptr;
    float2* twa = nullptr;
    float2* twb = nullptr;
    float2* sa = nullptr;   // sub-band pass A: sa[b][m1] = W_32768^(b m1)
    float2* sb = nullptr;   //                  sb[b][m2] = W_1024^(b m2)   (b, m1, m2 < 32)
};
std::mutex g_fft_mu;
std::vector<FftTables> g_fft_tables;

bfs_status fft_tables(FftTables* out) {
    int dev = 0;
    BFS_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(g_fft_mu);
    if (static_cast<int>(g_fft_tables.size()) <= dev) g_fft_tables.resize(dev + 1);
    FftTables& t = g_fft_tables[dev];
    if (!t.twa) {
        const double pi = 3.14159265358979323846;
        auto w = [&](long long num, long long den) {
            const double ph = -2.0 * pi * static_cast<double>(num % den) / static_cast<double>(den);
            return make_float2(static_cast<float>(std::cos(ph)), static_cast<float>(std::sin(ph)));
        };
        std::vector<float2> sm(64), a(kF * 32), b(kF * 32), sa(32 * 32), sb(32 * 32);
        for (int q = 0; q < 32; ++q) { sm[q] = w(q, 32); sm[32 + q] = w(q, kF); }
        for (long long n2 = 0; n2 < kF; ++n2)
            for (long long m = 0; m < 32; ++m) {
                a[n2 * 32 + m] = w(n2 * m, kFftN);
                b[n2 * 32 + m] = w(32 * n2 * m, kFftN);
            }
        for (long long bb = 0; bb < 32; ++bb)
            for (long long m = 0; m < 32; ++m) {
                sa[bb * 32 + m] = w(bb * m, kSubN);
                sb[bb * 32 + m] = w(bb * m, kF);
            }
        float2* d = nullptr;
        const size_t n = sm.size() + a.size() + b.size() + sa.size() + sb.size();
        BFS_CUDA(cudaMalloc(&d, n * sizeof(float2)));
        size_t off = 0;
        cudaError_t e = cudaSuccess;
        for (const std::vector<float2>* v : {&sm, &a, &b, &sa, &sb}) {
            if (e == cudaSuccess) e = cudaMemcpy(d + off, v->data(), v->size() * sizeof(float2), cudaMemcpyHostToDevice);
            off += v->size();
        }
        if (e != cudaSuccess) { cudaFree(d); return fail(BFS_ERR_CUDA, "FFT twiddle upload: %s", cudaGetErrorString(e)); }
        t.small = d;
        t.twa = d + 64;
        t.twb = t.twa + a.size();
        t.sa = t.twb + b.size();
        t.sb = t.sa + sa.size();
    }
    *out = t;
    return BFS_OK;
}

template <typename K>
bfs_status smem_opt_in(K kern, size_t bytes) {
    static std::mutex mu;
    static std::vector<std::pair<const void*, int>> done;
    int dev = 0;
    BFS_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    for (const auto& d : done)
        if (d.first == reinterpret_cast<const void*>(kern) && d.second == dev) return BFS_OK;
    BFS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)));
    done.emplace_back(reinterpret_cast<const void*>(kern), dev);
    return BFS_OK;
}

}  // namespace

bool fft_fused_supported(int nbin, int npol) { return nbin == kFftN && (npol == 2 || npol == 4); }

// The own sub-band transforms: mbin = nbin / len_sft = 32768, nbin a power of
// two, one or two polarisations.
bool subband_ifft_supported(int nbin, int len_sft, int npol) {
    return len_sft >= 1 && nbin % len_sft == 0 && nbin / len_sft == kSubN && (nbin & (nbin - 1)) == 0 &&
           (npol == 2 || npol == 4);
}

// Inverse transforms of every chirped sub-band of spec (complex64
// [pol][fft][chan][nbin], 16-byte aligned) with the chirp table chirp
// ([chan][sub-band][mbin], 16-byte aligned): plane == nullptr -> the voltages
// in z (same layout as spec); else z is scratch and the detected,
// dedispersed plane (rows x msamp) goes to plane, shift = the rows' shifts.
bfs_status subband_ifft(const float2* spec, const float2* chirp, float2* z, float* plane, const int* shift,
                        int npol2, int nfft, int nchan, int len_sft, int nbin, int nov_pc, int mbin_adj, int msamp,
                        cudaStream_t s) {
    FftTables t;
    bfs_status st = fft_tables(&t);
    if (st != BFS_OK) return st;
    BFS_ARG(subband_ifft_supported(nbin, len_sft, 2 * npol2), "no own sub-band transform for this geometry");
    BFS_ARG(reinterpret_cast<uintptr_t>(spec) % 16 == 0 && reinterpret_cast<uintptr_t>(chirp) % 16 == 0,
            "spectrum and chirp table must be 16-byte aligned");
    const long long nseg = static_cast<long long>(npol2) * nfft;
    const long long nsub = static_cast<long long>(nchan) * len_sft;
    const long long ga = nseg * (32 / kSubCols) * nsub;
    BFS_ARG(ga < (1ll << 31), "too many sub-bands");
    st = smem_opt_in(k_subfft_cols, kSubColSmem);
    if (st != BFS_OK) return st;
    k_subfft_cols<<<static_cast<unsigned>(ga), 32 * kSubCols, kSubColSmem, s>>>(
        spec, chirp, z, t.small, t.sa, t.sb, static_cast<int>(nseg), nchan, len_sft, nbin);
    BFS_LAUNCH_CHECK("k_subfft_cols");
    const double inv_nbin2 = 1.0 / (static_cast<double>(nbin) * nbin);   // exact: nbin is a power of two
    const int kBlk = kF / kSubRowThreads;
    if (plane) {
        const long long gb = kBlk * static_cast<long long>(nfft) * nsub;
        BFS_ARG(gb < (1ll << 31), "too many sub-bands");
        k_subfft_rows<true><<<static_cast<unsigned>(gb), kSubRowThreads, 0, s>>>(
            z, plane, shift, npol2, nfft, nchan, len_sft, nbin, nov_pc, mbin_adj, msamp, inv_nbin2);
    } else {
        const long long gb = kBlk * nseg * nsub;
        BFS_ARG(gb < (1ll << 31), "too many sub-bands");
        k_subfft_rows<false><<<static_cast<unsigned>(gb), kSubRowThreads, 0, s>>>(
            z, nullptr, nullptr, npol2, nfft, nchan, len_sft, nbin, nov_pc, mbin_adj, msamp, inv_nbin2);
    }
    BFS_LAUNCH_CHECK("k_subfft_rows");
    return BFS_OK;
}

// x (segments of kFftN complex, [pol][fft][chan]) = forward FFT of the
// unpacked int8 chunk raw; tmp holds the column-pass result (same size).
bfs_status fft_forward_guppi(const signed char* raw, float2* tmp, float2* x, long long nsamp, int noverlap,
                             int nfft, int nchan, int npol, cudaStream_t s) {
    FftTables t;
    bfs_status st = fft_tables(&t);
    if (st != BFS_OK) return st;
    BFS_ARG(nfft <= 65535 && nchan <= 65535, "too many segments or channels");
    dim3 gc(kF / kColCols, nfft, nchan);
    if (npol == 4) {
        st = smem_opt_in(k_fft_cols_guppi<2>, kColSmem(2));
        if (st != BFS_OK) return st;
        k_fft_cols_guppi<2><<<gc, 32 * 2 * kColCols, kColSmem(2), s>>>(raw, tmp, t.small, t.twa, t.twb, nsamp,
                                                                        noverlap, nfft, nchan);
    } else {
        st = smem_opt_in(k_fft_cols_guppi<1>, kColSmem(1));
        if (st != BFS_OK) return st;
        k_fft_cols_guppi<1><<<gc, 32 * kColCols, kColSmem(1), s>>>(raw, tmp, t.small, t.twa, t.twb, nsamp,
                                                                    noverlap, nfft, nchan);
    }
    BFS_LAUNCH_CHECK("k_fft_cols_guppi");
    const long long nseg = static_cast<long long>(npol / 2) * nfft * nchan;
    BFS_ARG(nseg <= 65535, "too many segments");
    st = smem_opt_in(k_fft_rows, kRowSmem);
    if (st != BFS_OK) return st;
    k_fft_rows<<<dim3(kF / kRowRows, static_cast<unsigned>(nseg)), 32 * kRowRows, kRowSmem, s>>>(tmp, x, t.small);
    BFS_LAUNCH_CHECK("k_fft_rows");
    return BFS_OK;
}

}  // namespace bfs
