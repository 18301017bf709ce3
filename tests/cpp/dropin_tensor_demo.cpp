// A reference-style driver on the tensor-core path: use_tensor_cores(true)
// before MSOSM_GPU_DM_concurrent / MSOSM_GPU_BATCH are initialised, then the
// reference's calls (initialize_uint16, filter_block_uint16, get_output,
// synchronize).  argv: fftpoint, input file of uint16 pairs, output file.
// Writes, per call, the concurrent object's trials then the single-DM
// object's series as raw complex64.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "msosm_gpu_b200.hpp"

using namespace msosm_b200;

int main(int argc, char **argv)
{
    if (argc != 4)
        return 2;
    const unsigned long fftpoint = std::strtoul(argv[1], nullptr, 10);
    const int calls = 3, count = 2;
    const unsigned long M = fftpoint / 2, blk = count * M;
    std::vector<uint16_pair> in(blk * calls);
    FILE *f = std::fopen(argv[2], "rb");
    if (!f || std::fread(in.data(), sizeof(uint16_pair), in.size(), f) != in.size())
        return 3;
    std::fclose(f);
    FILE *out = std::fopen(argv[3], "wb");
    if (!out)
        return 3;
    float bw[3] = {16e6f, 16e6f, 16e6f}, dm[3] = {0.5f, 20.0f, 60.0f}, f0[3] = {1242e6f, 1242e6f, 1242e6f};

    use_tensor_cores(true);
    MSOSM_GPU_DM_concurrent conc(bw, dm, f0, 3);
    conc.initialize_uint16(fftpoint, count, 0, true);
    MSOSM_GPU_BATCH single(16e6f, 20.0f, 1242e6f);
    single.initialize_uint16(fftpoint, count);
    use_tensor_cores(false);
    if (conc.M_common != M || single.count != count)
        return 4;

    std::vector<Complex> o(3 * blk + 1), s(blk);
    for (int c = 0; c < calls; ++c) {
        conc.filter_block_uint16(in.data() + c * blk);
        conc.get_output(o.data());
        conc.synchronize();
        single.filter_block_uint16(in.data() + c * blk);
        single.get_output(s.data());
        std::fwrite(o.data(), sizeof(Complex), 3 * blk, out);
        std::fwrite(s.data(), sizeof(Complex), blk, out);
    }
    std::fclose(out);
    return 0;
}
