// A reference-style session driver (the GUPPI GPU branch of the reference's
// my_hcdmt_inwork/main.cpp: CSession_guppi_gpu + launch), compiled with
// include/bfs_dropin.hpp instead of the reference headers.
//   session_demo <guppi file> <images.bin> <t_p> <d_min> <d_max> <sigma> <nbin> <nfft>
// Runs CSession_guppi_gpu::launch (the delegate log goes to candidates.log in
// the working directory), writes the last chunk's images (one max_dt x msamp
// float32 plane per coherent DM) and prints
// "msamp ndm len_sft noverlap ncoherent len_chunk".
#include <cstdio>
#include <string>
#include <vector>

#include "bfs_dropin.hpp"

int main(int argc, char** argv) {
    if (argc != 9) {
        std::fprintf(stderr, "usage: %s guppi images t_p d_min d_max sigma nbin nfft\n", argv[0]);
        return 2;
    }
    CSession_guppi_gpu session(argv[1], ".", std::stof(argv[3]), std::stod(argv[4]), std::stod(argv[5]),
                               std::stof(argv[6]), 1, std::stoi(argv[7]), std::stoi(argv[8]));
    std::vector<std::vector<float>> vecImg;
    int msamp = 0;
    if (-1 == session.launch(&vecImg, &msamp)) return 3;
    FILE* f = std::fopen(argv[2], "wb");
    if (!f) return 4;
    for (const std::vector<float>& img : vecImg) std::fwrite(img.data(), sizeof(float), img.size(), f);
    std::fclose(f);
    const bfs_guppi_session& p = session.m_plan;
    std::printf("%d %zu %d %d %d %lld\n", msamp, vecImg.size(), p.len_sft, p.noverlap, p.ncoherent,
                static_cast<long long>(p.len_chunk));
    return 0;
}
