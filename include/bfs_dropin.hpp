// bfs_dropin.hpp — header-only C++ shims with the reference's own names and
// signatures, implemented on the C ABI in bfs.h.  A reference call site keeps
// compiling unchanged: include this header instead of FdmtGpu.cuh,
// Statistical_preprocessing.cuh and Clusterization.cuh, and link libbfs_b200.
//
//   CFdmtGpu                      L/FDMT/FdmtGpu.cuh:5-53
//   FDMTGPU (Pravir plan)         L/FDMT_PRAVIR/fdmt_base.hpp:37-84, fdmt_gpu.cuh
//   COutChunkHeader               L/OutChunkHeader.h, OutChunkHeader.cpp:89-227
//   CFragment, cutQuadraticFragment  L/Fragment.h:3-28, L/CDMT/ChunkB.cpp:255-275
//   statistical_preprocessing::   L/CDMT/Statistical_preprocessing.cuh:9-10
//   clusterization::              L/Clusterization/Clusterization.cuh:10-67
//   select_delegates::write_log   L/Clusterization/select_delegates.cu:127-177
// (L = MyVSLib_C++).  As in the reference, pointers are device pointers,
// work runs on the default stream and errors are printed to stderr; the
// extra last_status() reports the bfs_status of the last call.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <fstream>
#include <iomanip>
#include <stdexcept>
#include <string>
#include <vector>

#include "bfs.h"

#ifndef fdmt_type_
#define fdmt_type_ float
#endif

using Cand = bfs_cand;  // same 16-byte layout as the reference's SCand

namespace bfs_dropin_detail {
inline bfs_status report(bfs_status st, const char* where) {
    if (st != BFS_OK) std::fprintf(stderr, "%s failed: %s\n", where, bfs_last_error());
    return st;
}
}  // namespace bfs_dropin_detail

class CFdmtGpu {
public:
    CFdmtGpu() = default;
    CFdmtGpu(const float Fmin, const float Fmax, int nchan, const int cols, int imaxDt)
        : m_nchan(nchan), m_cols(cols), m_Fmin(Fmin), m_Fmax(Fmax), m_imaxDt(imaxDt) {
        bfs_fdmt_desc d{};
        d.fmin = Fmin; d.fmax = Fmax; d.nchan = nchan; d.ncols = cols; d.max_dt = imaxDt;
        d.plan_kind = BFS_PLAN_KEITH; d.precision = BFS_PREC_F32; d.fuse_depth = -1;
        m_status = bfs_dropin_detail::report(bfs_fdmt_plan_create(&d, &m_plan), "CFdmtGpu");
        if (m_plan) {
            bfs_fdmt_info info{};
            bfs_fdmt_plan_info(m_plan, &info);
            m_iNumIter = info.niter;
        }
    }
    CFdmtGpu(const CFdmtGpu& R) : CFdmtGpu(R.m_Fmin, R.m_Fmax, R.m_nchan, R.m_cols, R.m_imaxDt) {}
    CFdmtGpu& operator=(const CFdmtGpu& R) {
        if (this != &R) {
            CFdmtGpu tmp(R);
            std::swap(m_plan, tmp.m_plan);
            m_nchan = R.m_nchan; m_cols = R.m_cols; m_Fmin = R.m_Fmin; m_Fmax = R.m_Fmax;
            m_imaxDt = R.m_imaxDt; m_iNumIter = R.m_iNumIter; m_status = tmp.m_status;
        }
        return *this;
    }
    ~CFdmtGpu() { if (m_plan) bfs_fdmt_plan_destroy(m_plan); }

    // d_parrImage: nchan x cols on the device; u_parrImOut: imaxDt x cols.
    void process_image(fdmt_type_* d_parrImage, fdmt_type_* u_parrImOut, const bool b_ones) {
        if (!m_plan) { m_status = BFS_ERR_ARG; std::fprintf(stderr, "CFdmtGpu: no plan\n"); return; }
        m_status = bfs_dropin_detail::report(
            bfs_fdmt_execute(m_plan, d_parrImage, u_parrImOut, b_ones ? 1 : 0, nullptr),
            "CFdmtGpu::process_image");
    }
    bfs_status last_status() const { return m_status; }

    int m_nchan = 0, m_cols = 0;
    float m_Fmin = 0, m_Fmax = 0;
    int m_imaxDt = 0, m_iNumIter = 0;

private:
    bfs_fdmt_plan* m_plan = nullptr;
    bfs_status m_status = BFS_OK;
};

// The reference's second FDMT variant (L/FDMT_PRAVIR/fdmt_base.hpp:37-84,
// fdmt_gpu.cuh): FDMTGPU(f_min, f_max, nchans, nsamps, tsamp, dt_max,
// dt_step, dt_min), execute(waterfall, waterfall_size, dmt, dmt_size) on
// device pointers, throwing std::invalid_argument on a size mismatch (as
// FDMT::check_inputs, fdmt_base.cpp:106-116) and std::runtime_error where the
// library reports an error.
class FDMTGPU {
public:
    FDMTGPU(float f_min, float f_max, size_t nchans, size_t nsamps, float tsamp, size_t dt_max,
            size_t dt_step = 1, size_t dt_min = 0)
        : m_nchans(nchans), m_nsamps(nsamps), m_tsamp(tsamp), m_f_min(f_min), m_f_max(f_max) {
        bfs_fdmt_desc d{};
        d.fmin = f_min; d.fmax = f_max; d.nchan = static_cast<int>(nchans);
        d.ncols = static_cast<int>(nsamps); d.max_dt = static_cast<int>(dt_max);
        d.plan_kind = BFS_PLAN_PRAVIR; d.precision = BFS_PREC_F32; d.fuse_depth = 0;
        d.dt_step = static_cast<int>(dt_step); d.dt_min = static_cast<int>(dt_min); d.tsamp = tsamp;
        if (bfs_fdmt_plan_create(&d, &m_plan) != BFS_OK) throw std::runtime_error(bfs_last_error());
        bfs_fdmt_info info{};
        bfs_fdmt_plan_info(m_plan, &info);
        m_niters = static_cast<size_t>(info.niter);
        m_dt_grid.resize(static_cast<size_t>(info.out_rows));
        std::vector<int> dt(m_dt_grid.size());
        bfs_fdmt_plan_delays(m_plan, dt.data(), static_cast<int>(dt.size()), nullptr, nullptr, 0);
        for (size_t i = 0; i < dt.size(); ++i) m_dt_grid[i] = static_cast<size_t>(dt[i]);
    }
    FDMTGPU(const FDMTGPU&) = delete;
    FDMTGPU& operator=(const FDMTGPU&) = delete;
    ~FDMTGPU() { if (m_plan) bfs_fdmt_plan_destroy(m_plan); }

    float get_df() const { return (m_f_max - m_f_min) / static_cast<float>(m_nchans); }
    float get_correction() const { return get_df() / 2; }
    size_t get_niters() const { return m_niters; }
    const std::vector<size_t>& get_dt_grid_final() const { return m_dt_grid; }
    std::vector<float> get_dm_grid_final() const {
        const float k = 4.1493774e3f;  // L/FDMT_PRAVIR/fdmtUtils.hpp:9,11
        const float conv = k * (std::pow(m_f_min, -2.0f) - std::pow(m_f_max, -2.0f));
        const float step = m_tsamp / conv;
        std::vector<float> dm(m_dt_grid.size());
        for (size_t i = 0; i < dm.size(); ++i) dm[i] = static_cast<float>(m_dt_grid[i]) * step;
        return dm;
    }
    void execute(const float* waterfall, size_t waterfall_size, float* dmt, size_t dmt_size) {
        if (waterfall_size != m_nchans * m_nsamps) throw std::invalid_argument("Invalid size of waterfall");
        if (dmt_size != m_dt_grid.size() * m_nsamps) throw std::invalid_argument("Invalid size of dmt");
        if (bfs_fdmt_execute(m_plan, waterfall, dmt, 0, nullptr) != BFS_OK)
            throw std::runtime_error(bfs_last_error());
    }

private:
    bfs_fdmt_plan* m_plan = nullptr;
    size_t m_nchans, m_nsamps, m_niters = 0;
    float m_tsamp, m_f_min, m_f_max;
    std::vector<size_t> m_dt_grid;
};

// Candidate report line and writer (L/OutChunkHeader.h, OutChunkHeader.cpp:89-227).
class COutChunkHeader {
public:
    COutChunkHeader() = default;
    COutChunkHeader(int nrows, int ncols, int nSucessRow, int nSucessCol, int width, float SNR,
                    float coherentDedisp, int numBlock, int numChunk)
        : m_nrows(nrows), m_ncols(ncols), m_nSucessRow(nSucessRow), m_nSucessCol(nSucessCol),
          m_SNR(SNR), m_coherentDedisp(coherentDedisp), m_numBlock(numBlock), m_numChunk(numChunk),
          m_wnd_width(width) {}
    int m_nrows = 0, m_ncols = 0, m_nSucessRow = 0, m_nSucessCol = 0;
    float m_SNR = 0, m_coherentDedisp = 0;
    int m_numBlock = 0, m_numChunk = 0, m_wnd_width = 0;

    void createOutStr(char* pstr) const {
        std::sprintf(pstr, "Block=  %d,Chunk=  %d,Rows=  %d,Cols=  %d, SucRow=  %d,SucCol=  %d, SNR=  %.4f, "
                     "CohDisp=  %.4f, windWidth=  %d", m_numBlock + 1, m_numChunk + 1, m_nrows, m_ncols,
                     m_nSucessRow, m_nSucessCol, m_SNR, m_coherentDedisp, m_wnd_width);
    }
    static void writeReport(const char* path, std::vector<COutChunkHeader>* headers, const float pulse_length) {
        FILE* f = std::fopen(path, "wb");
        if (!f) { std::printf("Can not open output file for writing"); return; }
        for (const COutChunkHeader& h : *headers) {
            char line[400] = {0};
            h.createOutStr(line);
            std::fprintf(f, "%s, Length of pulse= %.10e\n", line, pulse_length);
        }
        std::fclose(f);
    }
};

// Square cut-out around a detection (L/Fragment.h:3-28) and the cut rule of
// CChunkB::cutQuadraticFragment (L/CDMT/ChunkB.cpp:255-275) on a device plane.
class CFragment {
public:
    CFragment() = default;
    CFragment(const float* parr, int IDim, int NBeginRow, int NBeginCol, int NWidth, float VAlsnr, float cohDisp)
        : m_nBeginRow(NBeginRow), m_nBeginCol(NBeginCol), m_dim(IDim),
          m_vctData(parr, parr + static_cast<size_t>(IDim) * IDim), m_width(NWidth), m_snr(VAlsnr),
          m_cohDisp(cohDisp) {}
    int m_nBeginRow = 0, m_nBeginCol = 0, m_dim = 0;
    std::vector<float> m_vctData = std::vector<float>(1);
    int m_width = 0;
    float m_snr = 0, m_cohDisp = 0;
};

// parrFragment: device buffer of min(rows, cols)^2 floats; parrInpImage: device plane.
inline void cutQuadraticFragment(float* parrFragment, float* parrInpImage, int* piRowBegin, int* piColBegin,
                                 const int QInpImageRows, const int QInpImageCols, const int NUmTargetRow,
                                 const int NUmTargetCol) {
    int dim = 0;
    bfs_dropin_detail::report(bfs_cut_fragment(parrInpImage, QInpImageRows, QInpImageCols, NUmTargetRow,
                                               NUmTargetCol, parrFragment, piRowBegin, piColBegin, &dim,
                                               nullptr),
                              "cutQuadraticFragment");
}

namespace statistical_preprocessing {
inline void calc_fdmt_inputs(float* d_parr_inp, const int NRows, const int NCols, float* d_buff,
                             float* d_parrNormInput) {
    bfs_dropin_detail::report(
        bfs_preproc_calc_fdmt_inputs(d_parr_inp, NRows, NCols, d_buff, d_parrNormInput, nullptr),
        "calc_fdmt_inputs");
}
}  // namespace statistical_preprocessing

namespace select_delegates {
// Delegate log, the reference's columns and widths.  h_delegates are
// candidate indices sorted by mt; h_offsets the group starts (ngroups + 1).
inline void write_log(const std::vector<Cand>& h_cands, const std::vector<int>& h_offsets,
                      const std::vector<int>& h_delegates, const std::string& filename,
                      const float delt_bin, const float t_chunkBegin) {
    std::ofstream log(filename);
    log << std::setw(10) << "N" << std::setw(10) << "t, bin" << std::setw(10) << "t, sec"
        << std::setw(10) << "dedisp" << std::setw(10) << "width" << std::setw(10) << "SNR"
        << std::setw(10) << "num" << std::endl;
    for (size_t i = 0; i < h_delegates.size(); ++i) {
        const Cand c = h_cands[h_delegates[i]];
        // the reference pairs the i-th delegate with the i-th group's size
        const int num = h_offsets[i + 1] - h_offsets[i];
        log << std::setw(10) << i + 1 << std::setw(10) << c.mt << std::setw(10)
            << t_chunkBegin + c.mt * delt_bin << std::setw(10) << c.mdt << std::setw(10)
            << c.mwidth << std::setw(10) << c.msnr << std::setw(10) << num << std::endl;
    }
}
}  // namespace select_delegates

namespace clusterization {

// Boxcar gather into a freshly cudaMalloc'd array the caller frees (the
// reference's ownership rule).  val_thresh is a reference to device memory.
inline bool gather_(const float* d_plane, int Rows, int Cols, const float& val_thresh, int mode,
                    int param, Cand** d_out, unsigned int* h_count) {
    *d_out = nullptr;
    *h_count = 0;
    uint32_t cap = 1u << 16, n = 0;
    for (int attempt = 0; attempt < 2; ++attempt) {
        Cand* buf = nullptr;
        if (cudaMalloc(reinterpret_cast<void**>(&buf), sizeof(Cand) * (cap ? cap : 1)) != cudaSuccess) {
            std::fprintf(stderr, "gather: cudaMalloc failed\n");
            return false;
        }
        const bfs_status st = bfs_boxcar_gather(d_plane, Rows, Cols, nullptr, 0.0f, &val_thresh, mode,
                                                param, 0, buf, cap, &n, nullptr);
        if (st == BFS_OK) { *d_out = buf; *h_count = n; return true; }
        cudaFree(buf);
        if (st != BFS_ERR_OVERFLOW) { bfs_dropin_detail::report(st, "gather"); return false; }
        cap = n;  // retry with the exact count
    }
    return false;
}

inline void gather_candidates_in_dynamicalArray(const float* d_arr_fdmt, const int Rows, const int Cols,
                                                const float& val_thresh, const int QUantPower2_Wnd,
                                                Cand** d_arrCand, unsigned int* h_pquantCand) {
    gather_(d_arr_fdmt, Rows, Cols, val_thresh, BFS_WIDTHS_POW2, QUantPower2_Wnd, d_arrCand,
            h_pquantCand);
}

inline bool gather_candidates_in_heap_with_plan(const float* d_fdmt, const int Rows, const int Cols,
                                                const float& d_VAlTresh, const int WndWidth,
                                                Cand** d_pparrCand, unsigned int* h_piQuantCand) {
    return gather_(d_fdmt, Rows, Cols, d_VAlTresh, BFS_WIDTHS_ALL, WndWidth, d_pparrCand,
                   h_piQuantCand) && *h_piQuantCand > 0;
}

// d_pbin_metrics: 3 ints in device memory (as in the reference).
inline void complete_clusterization(const Cand* d_parrCand, unsigned int quant_candidates,
                                    const int* d_pbin_metrics, const std::string& filename,
                                    const float delt_bin, const float t_chunkBegin, bool bwrite) {
    if (quant_candidates == 0) return;
    int metrics[3];
    cudaMemcpy(metrics, d_pbin_metrics, sizeof(metrics), cudaMemcpyDeviceToHost);
    int *perm = nullptr, *offsets = nullptr, *dl = nullptr;
    cudaMalloc(reinterpret_cast<void**>(&perm), sizeof(int) * quant_candidates);
    cudaMalloc(reinterpret_cast<void**>(&offsets), sizeof(int) * (quant_candidates + 1));
    cudaMalloc(reinterpret_cast<void**>(&dl), sizeof(int) * quant_candidates);
    uint32_t ng = 0;
    const bfs_status st = bfs_cluster(d_parrCand, quant_candidates, metrics, perm, offsets, dl, &ng,
                                      nullptr);
    if (bfs_dropin_detail::report(st, "complete_clusterization") == BFS_OK && bwrite) {
        std::vector<Cand> c(quant_candidates);
        std::vector<int> o(ng + 1), d(ng);
        cudaMemcpy(c.data(), d_parrCand, sizeof(Cand) * quant_candidates, cudaMemcpyDeviceToHost);
        cudaMemcpy(o.data(), offsets, sizeof(int) * (ng + 1), cudaMemcpyDeviceToHost);
        cudaMemcpy(d.data(), dl, sizeof(int) * ng, cudaMemcpyDeviceToHost);
        select_delegates::write_log(c, o, d, filename, delt_bin, t_chunkBegin);
    }
    cudaFree(perm);
    cudaFree(offsets);
    cudaFree(dl);
}

inline bool clusterization_main(const float* d_digitized_fdmt, const int Rows, const int Cols,
                                const float& d_VAlTresh, const int WndWidth,
                                const int* d_pbin_metrics, const std::string& filename,
                                const float delt_bin, const float t_chunkBegin, bool bwrite = true) {
    Cand* d_cands = nullptr;
    unsigned int n = 0;
    if (!gather_candidates_in_heap_with_plan(d_digitized_fdmt, Rows, Cols, d_VAlTresh, WndWidth,
                                             &d_cands, &n)) {
        if (d_cands) cudaFree(d_cands);
        return false;
    }
    complete_clusterization(d_cands, n, d_pbin_metrics, filename, delt_bin, t_chunkBegin, bwrite);
    cudaFree(d_cands);
    return true;
}

}  // namespace clusterization

// ---------------------------------------------------------------------------
// Coherent-dedispersion chunk and the GUPPI session driver.
//
//   CChunkB              L/CDMT/ChunkB.h:8-114 (geometry, DM grid ChunkB.cpp:171-176)
//   CChunk_gpu           L/CDMT/Chunk_gpu.cuh:16-72, Chunk_gpu.cu:254-460
//   CSession_guppi_gpu   L/CDMT/Session_guppi_gpu.cuh:9-39, SessionB.cpp:106-300
//
// CChunk_gpu::process takes the unpacked complex chunk (overwritten by the
// forward FFT), makes one normalised FDMT plane (len_sft x msamp) per
// coherent DM, runs clusterization_main on all of them (every width 1..4,
// threshold sigma_bound, splitters {2, 1, 2}, delegate log "candidates.log",
// delt_bin = tsamp * len_sft) and copies the planes to pvecImg, as the
// reference does.  The reference's discarded gather_candidates_in_
// dynamicalArray call and its unused success headers are left out.
// CSession_guppi_gpu::launch derives the chunk geometry from the first
// block's header (bfs_guppi_session_plan), streams every chunk of every block
// through pinned buffers to the device and calls CChunk_gpu::process_raw
// (unpack and forward FFT fused); it returns 0, or -1 on an error (the value
// the reference's drivers test for).
// ---------------------------------------------------------------------------
class CChunkB {
public:
    CChunkB() = default;
    CChunkB(const float Fmin, const float Fmax, const int npol, const int nchan, const unsigned int len_sft,
            const int Block_id, const int Chunk_id, const double d_max, const double d_min, const int ncoherent,
            const float sigma_bound, const int length_sum_wnd, const int nbin, const int nfft,
            const int noverlap, const float tsamp)
        : m_Fmin(Fmin), m_Fmax(Fmax), m_npol(npol), m_nchan(nchan), m_len_sft(len_sft), m_tsamp(tsamp),
          m_Chunk_id(Chunk_id), m_Block_id(Block_id), m_d_max(d_max), m_d_min(d_min), m_ncoherent(ncoherent),
          m_sigma_bound(sigma_bound), m_length_sum_wnd(length_sum_wnd), m_nbin(nbin), m_nfft(nfft),
          m_noverlap(noverlap) {
        const int n = bfs_chunk_coherent_dms(d_min, d_max, ncoherent, nullptr, 0);
        m_coh_dm_Vector.resize(static_cast<size_t>(n > 0 ? n : 0));
        if (n > 0) bfs_chunk_coherent_dms(d_min, d_max, ncoherent, m_coh_dm_Vector.data(), n);
    }
    virtual ~CChunkB() = default;

    float m_Fmin = 0, m_Fmax = 0;
    unsigned int m_npol = 0, m_nchan = 0, m_len_sft = 1;
    float m_tsamp = 0;
    int m_Chunk_id = 0, m_Block_id = 0;
    double m_d_max = 0, m_d_min = 0;
    int m_ncoherent = 0;
    float m_sigma_bound = 0;
    int m_length_sum_wnd = 0, m_nbin = 0, m_nfft = 0, m_noverlap = 0;
    std::vector<double> m_coh_dm_Vector;

    virtual bool process(void* /*pcmparrRawSignalCur*/, std::vector<COutChunkHeader>* /*pvctSuccessHeaders*/,
                         std::vector<std::vector<float>>* /*pvecImg*/) {
        return false;
    }
    int get_noverlap_per_channel() const { return m_noverlap / static_cast<int>(m_len_sft); }
    int get_mbin() const { return m_nbin / static_cast<int>(m_len_sft); }
    int get_mbin_adjusted() const { return get_mbin() - 2 * get_noverlap_per_channel(); }
    int get_msamp() const { return m_nfft * get_mbin_adjusted(); }
    void set_chunkid(const int nC) { m_Chunk_id = nC; }
    void set_blockid(const int nC) { m_Block_id = nC; }
    static void cutQuadraticFragment(float* parrFragment, float* parrInpImage, int* piRowBegin, int* piColBegin,
                                     const int QInpImageRows, const int QInpImageCols, const int NUmTargetRow,
                                     const int NUmTargetCol) {
        ::cutQuadraticFragment(parrFragment, parrInpImage, piRowBegin, piColBegin, QInpImageRows, QInpImageCols,
                               NUmTargetRow, NUmTargetCol);
    }
};

class CChunk_gpu : public CChunkB {
public:
    CChunk_gpu(const float Fmin, const float Fmax, const int npol, const int nchan, const unsigned int len_sft,
               const int Block_id, const int Chunk_id, const float d_max, const float d_min, const int ncoherent,
               const float sigma_bound, const int length_sum_wnd, const int nbin, const int nfft,
               const int noverlap, const float tsamp)
        : CChunkB(Fmin, Fmax, npol, nchan, len_sft, Block_id, Chunk_id, d_max, d_min, ncoherent, sigma_bound,
                  length_sum_wnd, nbin, nfft, noverlap, tsamp) {
        bfs_chunk_desc d{};
        d.fmin = Fmin; d.fmax = Fmax; d.npol = npol; d.nchan = nchan; d.len_sft = static_cast<int>(len_sft);
        d.nbin = nbin; d.nfft = nfft; d.noverlap = noverlap; d.tsamp = tsamp; d.max_dt = 0;
        m_status = bfs_dropin_detail::report(bfs_chunk_create(&d, &m_chunk), "CChunk_gpu");
        if (!m_chunk) return;
        int64_t info[8] = {0};
        bfs_chunk_info(m_chunk, info, 8);
        m_len_chunk = info[5];
        m_complex_values = info[6];
        m_max_dt = static_cast<int>(info[7]);
        // the threshold and the splitters live in device memory, as in the reference
        const int splitters[3] = {2, 1, 2};
        if (cudaMalloc(reinterpret_cast<void**>(&m_pd_thresh), sizeof(float)) != cudaSuccess ||
            cudaMalloc(reinterpret_cast<void**>(&m_pd_splitters), sizeof(splitters)) != cudaSuccess ||
            cudaMemcpy(m_pd_thresh, &m_sigma_bound, sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(m_pd_splitters, splitters, sizeof(splitters), cudaMemcpyHostToDevice) != cudaSuccess) {
            std::fprintf(stderr, "CChunk_gpu: device allocation failed\n");
            m_status = BFS_ERR_CUDA;
        }
    }
    CChunk_gpu(const CChunk_gpu&) = delete;
    CChunk_gpu& operator=(const CChunk_gpu&) = delete;
    ~CChunk_gpu() override {
        if (m_chunk) bfs_chunk_destroy(m_chunk);
        cudaFree(m_pdoutImg);
        cudaFree(m_pd_thresh);
        cudaFree(m_pd_splitters);
    }

    // pcmparrRawSignalCur: the unpacked chunk, complex [npol/2][nfft][nchan][nbin] on the device.
    bool process(void* pcmparrRawSignalCur, std::vector<COutChunkHeader>* pvctSuccessHeaders,
                 std::vector<std::vector<float>>* pvecImg) override {
        (void)pvctSuccessHeaders;
        if (!ready()) return false;
        const bfs_status st = bfs_chunk_process(m_chunk, pcmparrRawSignalCur, m_coh_dm_Vector.data(),
                                                static_cast<int>(m_coh_dm_Vector.size()), m_pdoutImg, nullptr);
        if (bfs_dropin_detail::report(st, "CChunk_gpu::process") != BFS_OK) return false;
        return search_and_copy(pvecImg);
    }
    // process from the int8 GUPPI chunk [nchan][len_chunk][npol] (no reference
    // counterpart: unpack and forward FFT in one step); d_spec (complex_values()
    // complex numbers) receives the spectra.
    bool process_raw(const int8_t* d_raw, void* d_spec, std::vector<COutChunkHeader>* pvctSuccessHeaders,
                     std::vector<std::vector<float>>* pvecImg) {
        (void)pvctSuccessHeaders;
        if (!ready()) return false;
        const bfs_status st = bfs_chunk_process_raw(m_chunk, d_raw, d_spec, m_coh_dm_Vector.data(),
                                                    static_cast<int>(m_coh_dm_Vector.size()), m_pdoutImg, nullptr);
        if (bfs_dropin_detail::report(st, "CChunk_gpu::process_raw") != BFS_OK) return false;
        return search_and_copy(pvecImg);
    }
    // unpack_chunk_guppi_gpu (Session_guppi_gpu.cu:53-60,117-141) into d_cplx.
    bool unpack(const int8_t* d_raw, void* d_cplx) {
        return m_chunk && bfs_dropin_detail::report(bfs_chunk_unpack(m_chunk, d_raw, d_cplx, nullptr),
                                                    "CChunk_gpu::unpack") == BFS_OK;
    }
    int64_t len_chunk() const { return m_len_chunk; }
    int64_t complex_values() const { return m_complex_values; }
    int max_dt() const { return m_max_dt; }
    bfs_status last_status() const { return m_status; }

    std::string m_logfile = "candidates.log";  // the reference's fixed log name
    float* m_pdoutImg = nullptr;               // planes of every coherent DM, max_dt x msamp each

private:
    bool ready() {
        if (!m_chunk || m_status != BFS_OK) { std::fprintf(stderr, "CChunk_gpu: not created\n"); return false; }
        if (m_coh_dm_Vector.empty()) { std::fprintf(stderr, "CChunk_gpu: no coherent DM\n"); return false; }
        if (!m_pdoutImg) {
            const size_t n = m_coh_dm_Vector.size() * static_cast<size_t>(m_max_dt) * get_msamp();
            if (cudaMalloc(reinterpret_cast<void**>(&m_pdoutImg), n * sizeof(float)) != cudaSuccess) {
                std::fprintf(stderr, "CChunk_gpu: cudaMalloc of the output planes failed\n");
                m_pdoutImg = nullptr;
                return false;
            }
        }
        return true;
    }
    bool search_and_copy(std::vector<std::vector<float>>* pvecImg) {
        const int ndm = static_cast<int>(m_coh_dm_Vector.size());
        const int msamp = get_msamp();
        clusterization::clusterization_main(m_pdoutImg, m_max_dt * ndm, msamp, *m_pd_thresh, 4, m_pd_splitters,
                                            m_logfile, m_tsamp * static_cast<float>(m_len_sft), 0.0f);
        if (pvecImg) {
            const size_t plane = static_cast<size_t>(m_max_dt) * msamp;
            pvecImg->resize(static_cast<size_t>(ndm));
            for (int i = 0; i < ndm; ++i) {
                (*pvecImg)[i].resize(plane);
                if (cudaMemcpy((*pvecImg)[i].data(), m_pdoutImg + static_cast<size_t>(i) * plane,
                               plane * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
                    return false;
            }
        }
        return true;
    }

    bfs_chunk* m_chunk = nullptr;
    bfs_status m_status = BFS_OK;
    int64_t m_len_chunk = 0, m_complex_values = 0;
    int m_max_dt = 0;
    float* m_pd_thresh = nullptr;
    int* m_pd_splitters = nullptr;
};

class CSession_guppi_gpu {
public:
    CSession_guppi_gpu(const char* strGuppiPath, const char* strOutPutPath, const float t_p, const double d_min,
                       const double d_max, const float sigma_bound, const int length_sum_wnd, const int nbin,
                       const int nfft)
        : m_strInpPath(strGuppiPath), m_strOutPutPath(strOutPutPath), m_pulse_length(t_p), m_d_max(d_max),
          m_d_min(d_min), m_sigma_bound(sigma_bound), m_length_sum_wnd(length_sum_wnd), m_nbin(nbin),
          m_nfft(nfft) {}

    std::string m_strInpPath, m_strOutPutPath;
    float m_pulse_length;
    double m_d_max, m_d_min;
    float m_sigma_bound;
    int m_length_sum_wnd, m_nbin, m_nfft;
    std::vector<COutChunkHeader> m_vctSuccessHeaders;   // unused, as in the reference
    bfs_guppi_session m_plan{};                         // geometry of the last launch

    int launch(std::vector<std::vector<float>>* pvecImg, int* pmsamp) {
        using bfs_dropin_detail::report;
        bfs_guppi_file* f = nullptr;
        if (report(bfs_guppi_open(m_strInpPath.c_str(), &f), "CSession_guppi_gpu::launch") != BFS_OK) return -1;
        bfs_guppi_header h{};
        bfs_guppi_block_header(f, 0, &h);
        if (report(bfs_guppi_session_plan(&h, m_pulse_length, m_d_min, m_d_max, m_nbin, m_nfft, &m_plan),
                   "CSession_guppi_gpu::launch") != BFS_OK) {
            bfs_guppi_close(f);
            return -1;
        }
        int rc = -1;
        int8_t* d_raw = nullptr;
        void* d_spec = nullptr;
        bfs_guppi_reader* reader = nullptr;
        {
            CChunk_gpu chunk(m_plan.fmin, m_plan.fmax, h.npol, h.nchan, static_cast<unsigned>(m_plan.len_sft), 0, 0,
                             m_plan.d_max, m_plan.d_min, m_plan.ncoherent, m_sigma_bound, m_length_sum_wnd,
                             m_nbin, m_nfft, m_plan.noverlap, m_plan.tsamp);
            const size_t raw_bytes = static_cast<size_t>(h.nchan) * m_plan.len_chunk * h.npol;
            if (chunk.last_status() == BFS_OK &&
                cudaMalloc(reinterpret_cast<void**>(&d_raw), raw_bytes) == cudaSuccess &&
                cudaMalloc(&d_spec, static_cast<size_t>(chunk.complex_values()) * 2 * sizeof(float)) == cudaSuccess &&
                report(bfs_guppi_reader_create(f, m_plan.len_chunk, m_plan.noverlap, 2, 1, &reader),
                       "CSession_guppi_gpu::launch") == BFS_OK) {
                rc = 0;
                for (;;) {
                    int block = -1;
                    int64_t j = -1;
                    if (report(bfs_guppi_reader_next(reader, d_raw, nullptr, nullptr, &block, &j),
                               "CSession_guppi_gpu::launch") != BFS_OK) { rc = -1; break; }
                    if (block < 0) break;
                    chunk.set_blockid(block);
                    chunk.set_chunkid(static_cast<int>(j));
                    if (!chunk.process_raw(d_raw, d_spec, &m_vctSuccessHeaders, pvecImg)) { rc = -1; break; }
                    if (pmsamp) *pmsamp = chunk.get_msamp();
                }
            }
            if (reader) bfs_guppi_reader_destroy(reader);
        }
        cudaFree(d_raw);
        cudaFree(d_spec);
        bfs_guppi_close(f);
        return rc;
    }
};
