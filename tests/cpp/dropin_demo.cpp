// A reference-style driver written against the drop-in header: the same
// calls a program using MSOSM_GPU_DM_concurrent / MSOSM_GPU_BATCH /
// OSM_GPU_BATCH / MSOSM_GPU_BATCH_stream / MSOSM_GPU_DM_BATCH_loop makes
// (compare test_processing_speed_msosm_batch32_dm0to100.cpp:213-293).
// Reads uint16 pairs from argv[1], writes raw complex64 outputs of every
// class to argv[2] in the order listed below.
#include <cstdio>
#include <vector>

#include "msosm_gpu_b200.hpp"

using namespace msosm_b200;

int main(int argc, char **argv)
{
    if (argc != 3)
        return 2;
    const int calls = 4, count = 4;
    const unsigned long fftpoint = 1024, M = fftpoint / 2, blk = count * M;
    std::vector<uint16_pair> in(blk * calls);
    FILE *f = std::fopen(argv[1], "rb");
    if (!f || std::fread(in.data(), sizeof(uint16_pair), in.size(), f) != in.size())
        return 3;
    std::fclose(f);
    FILE *out = std::fopen(argv[2], "wb");
    float bw[3] = {16e6f, 16e6f, 16e6f}, dm[3] = {1.0f, 3.5f, 7.0f}, f0[3] = {1242e6f, 1242e6f, 1242e6f};

    MSOSM_GPU_DM_concurrent conc(bw, dm, f0, 3);
    conc.initialize_uint16(fftpoint, count, 0, true);
    std::vector<Complex> o(3 * blk + 1);
    for (int c = 0; c < calls; ++c) {
        conc.filter_block_uint16(in.data() + c * blk);
        conc.get_output(o.data());
        conc.synchronize();
        std::fwrite(o.data(), sizeof(Complex), 3 * blk, out);
    }

    MSOSM_GPU_BATCH single(16e6f, 3.5f, 1242e6f);
    single.initialize_uint16(fftpoint, count);
    std::vector<Complex> s(blk);
    for (int c = 0; c < calls; ++c) {
        single.filter_block_uint16(in.data() + c * blk);
        single.get_output(s.data());
        std::fwrite(s.data(), sizeof(Complex), blk, out);
    }

    // OSM raises the FFT to 2*next_power_of_2(Nd) when that exceeds fftpoint:
    // size everything from the object, as the reference drivers do
    OSM_GPU_BATCH osm(16e6f, 0.1f, 1242e6f);
    osm.initialize_uint16(fftpoint, count);
    const unsigned long oblk = (unsigned long)osm.count * osm.M;
    if (oblk > blk)
        return 4;
    std::vector<Complex> so(oblk);
    for (int c = 0; c < calls; ++c) {
        osm.filter_block_uint16(in.data() + c * oblk);
        osm.get_output(so.data());
        std::fwrite(so.data(), sizeof(Complex), oblk, out);
    }

    unsigned long fp[2] = {fftpoint, fftpoint};
    MSOSM_GPU_BATCH_stream streams(bw, dm, f0, 2);
    streams.initialize_uint16(fp, count);
    std::vector<Complex> s0(blk), s1(blk);
    Complex *outs[2] = {s0.data(), s1.data()};
    for (int c = 0; c < calls; ++c) {
        uint16_pair *ins[2] = {in.data() + c * blk, in.data() + c * blk};
        streams.filter_block_uint16(ins);
        streams.get_output(outs);
        streams.synchronize();
        std::fwrite(s0.data(), sizeof(Complex), blk, out);
        std::fwrite(s1.data(), sizeof(Complex), blk, out);
    }

    MSOSM_GPU_DM_BATCH_loop loop(bw, dm, f0, 3);
    loop.initialize_uint16(fftpoint, count);
    std::vector<Complex> l0(blk), l1(blk), l2(blk);
    Complex *louts[3] = {l0.data(), l1.data(), l2.data()};
    for (int c = 0; c < calls; ++c) {
        loop.input_process(in.data() + c * blk);
        for (int i = 0; i < 3; ++i)
            loop.filter_block_uint16(louts, i);
        loop.synchronize();
        for (int i = 0; i < 3; ++i)
            std::fwrite(louts[i], sizeof(Complex), blk, out);
    }
    std::fclose(out);
    return 0;
}
