// psrdada_demo.cpp -- the reference's msosm_psrdada driver
// (msosm_psrdada.cpp:92-144) written against the drop-in header: two
// MSOSM_GPU_BATCH (one per polarisation), Fold_GPU on the device, blank
// leading reads skipped, the profile written next to the file.
//
//   psrdada_demo <file.dada> <dm> <period> <fftpoint> <time_bin>
#include <cstdio>
#include <cstdlib>
#include <string>

#include "msosm_gpu_b200.hpp"

using namespace msosm_b200;

int main(int argc, char **argv)
{
    if (argc != 6) {
        std::fprintf(stderr, "usage: psrdada_demo <file.dada> <dm> <period> <fftpoint> <time_bin>\n");
        return 2;
    }
    const std::string filename = argv[1];
    const float dm = std::strtof(argv[2], nullptr), period = std::strtof(argv[3], nullptr);
    const unsigned long fftpoint = std::strtoul(argv[4], nullptr, 10), time_bin = std::strtoul(argv[5], nullptr, 10);
    const int count = 1;
    PSRDADA file(filename);
    float bw = file.bw, f0 = file.fc - bw / 2;
    bw = bw * 1e6f;
    f0 = f0 * 1e6f;
    MSOSM_GPU_BATCH msosm_gpu1(bw, dm, f0);
    MSOSM_GPU_BATCH msosm_gpu2(bw, dm, f0);
    msosm_gpu1.initialize_uint16(fftpoint, count);
    msosm_gpu2.initialize_uint16(fftpoint, count);
    const unsigned long M = msosm_gpu1.M;
    file.initBuffer(count * M);
    Fold_GPU fold(period, bw, count * M, file.outfileName, time_bin);
    fold.discard_samples(msosm_gpu1.Nd);
    bool first = true;
    for (unsigned long i = 0; i < file.readCount; i++) {
        file.readSamples();
        if (first) {
            if (file.pol1_in[0].first == 0)
                continue;
            first = false;
        }
        msosm_gpu1.filter_block_uint16(file.pol1_in);
        msosm_gpu2.filter_block_uint16(file.pol2_in);
        fold.calculate_intensity(&msosm_gpu1, &msosm_gpu2);
        fold.fold_data();
    }
    fold.fold_data_bins();
    fold.write_to_file();
    std::printf("folded %lu bins -> %s\n", fold.time_bin, file.outfileName.c_str());
    return 0;
}
