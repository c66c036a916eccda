// A reference-style driver written against the reference's own names
// (CFdmtGpu, clusterization::clusterization_main), compiled with
// include/bfs_dropin.hpp instead of the reference headers.
//   dropin_demo <fdmt_in.bin> <fdmt_out.bin> <log file> <pravir_out.bin>
// Reads a 64 x 1024 float32 filterbank, writes its FDMT (1200-1600 MHz,
// max delay 64), then runs clusterization_main on the reference's 3 x 16 test
// plane (clusterization_forpravir/clusterization_test.cu:63-112) with W = 2,
// threshold 4 and metrics {2, 1, 2}; also runs the Pravir-plan FDMTGPU
// (tsamp 1 ms, dt_max 64) on the same filterbank and checks that a size
// mismatch throws std::invalid_argument.
#include <cstdio>
#include <string>
#include <vector>

#include "bfs_dropin.hpp"

int main(int argc, char** argv) {
    if (argc != 5) { std::fprintf(stderr, "usage: %s in.bin out.bin log pravir.bin\n", argv[0]); return 2; }
    const int nchan = 64, cols = 1024, maxdt = 64;
    std::vector<float> in(nchan * cols), out(maxdt * cols);
    FILE* f = std::fopen(argv[1], "rb");
    if (!f || std::fread(in.data(), sizeof(float), in.size(), f) != in.size()) return 3;
    std::fclose(f);
    float *d_in = nullptr, *d_out = nullptr;
    cudaMalloc(reinterpret_cast<void**>(&d_in), in.size() * sizeof(float));
    cudaMalloc(reinterpret_cast<void**>(&d_out), out.size() * sizeof(float));
    cudaMemcpy(d_in, in.data(), in.size() * sizeof(float), cudaMemcpyHostToDevice);
    CFdmtGpu fdmt(1200.0f, 1600.0f, nchan, cols, maxdt);
    fdmt.process_image(d_in, d_out, false);
    cudaMemcpy(out.data(), d_out, out.size() * sizeof(float), cudaMemcpyDeviceToHost);
    if (fdmt.last_status() != BFS_OK) return 4;
    f = std::fopen(argv[2], "wb");
    std::fwrite(out.data(), sizeof(float), out.size(), f);
    std::fclose(f);

    {
        FDMTGPU pravir(1200.0f, 1600.0f, nchan, cols, 0.001f, maxdt);
        const size_t nout = pravir.get_dt_grid_final().size() * cols;
        float* d_pout = nullptr;
        cudaMalloc(reinterpret_cast<void**>(&d_pout), nout * sizeof(float));
        bool threw = false;
        try {
            pravir.execute(d_in, in.size() - 1, d_pout, nout);
        } catch (const std::invalid_argument&) {
            threw = true;
        }
        if (!threw) return 6;
        pravir.execute(d_in, in.size(), d_pout, nout);
        std::vector<float> pout(nout);
        cudaMemcpy(pout.data(), d_pout, nout * sizeof(float), cudaMemcpyDeviceToHost);
        cudaFree(d_pout);
        f = std::fopen(argv[4], "wb");
        std::fwrite(pout.data(), sizeof(float), pout.size(), f);
        std::fclose(f);
    }

    const int rows = 3, pc = 16;
    std::vector<float> plane(rows * pc, 2.0f);
    plane[4] = 140.0f; plane[11] = 120.0f; plane[2 * pc + 4] = 100.0f;
    float* d_plane = nullptr; float* d_thr = nullptr; int* d_metrics = nullptr;
    cudaMalloc(reinterpret_cast<void**>(&d_plane), plane.size() * sizeof(float));
    cudaMalloc(reinterpret_cast<void**>(&d_thr), sizeof(float));
    cudaMalloc(reinterpret_cast<void**>(&d_metrics), 3 * sizeof(int));
    const float thr = 4.0f; const int metrics[3] = {2, 1, 2};
    cudaMemcpy(d_plane, plane.data(), plane.size() * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(d_thr, &thr, sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(d_metrics, metrics, sizeof(metrics), cudaMemcpyHostToDevice);
    const bool found = clusterization::clusterization_main(d_plane, rows, pc, *d_thr, 2, d_metrics,
                                                           argv[3], 0.00001f, 0.0f);
    {
        // a report line for the brightest cell and its square fragment
        std::vector<COutChunkHeader> hdrs{COutChunkHeader(rows, pc, 0, 4, 1, 140.0f, 56.8f, 0, 0)};
        COutChunkHeader::writeReport((std::string(argv[3]) + ".report").c_str(), &hdrs, 1.25e-3f);
        float* d_frag = nullptr;
        cudaMalloc(reinterpret_cast<void**>(&d_frag), rows * rows * sizeof(float));
        int rb = -1, cb = -1;
        cutQuadraticFragment(d_frag, d_plane, &rb, &cb, rows, pc, 0, 4);
        std::vector<float> frag(rows * rows);
        cudaMemcpy(frag.data(), d_frag, frag.size() * sizeof(float), cudaMemcpyDeviceToHost);
        cudaFree(d_frag);
        const CFragment fr(frag.data(), rows, rb, cb, 1, 140.0f, 56.8f);
        if (fr.m_nBeginCol != 3 || fr.m_vctData[1] != 140.0f) return 7;
    }
    cudaFree(d_in); cudaFree(d_out); cudaFree(d_plane); cudaFree(d_thr); cudaFree(d_metrics);
    return found ? 0 : 5;
}
