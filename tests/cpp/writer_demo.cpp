// writer_demo.cpp -- the output-file driver of the reference
// (multiple_dm_concurrent_msosm.cpp:200-330: MSOSM_GPU_DM_concurrent over a
// simulated uint16 signal, every call's uint16 output appended to a file by
// a writer thread) written against the drop-in header: SeriesFileWriter
// replaces the thread, its busy-wait and get_output_thread.
//
//   writer_demo <numDMs> <count> <calls> <out.bin>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "msosm_gpu_b200.hpp"

using namespace msosm_b200;

int main(int argc, char **argv)
{
    if (argc != 5) {
        std::fprintf(stderr, "usage: writer_demo <numDMs> <count> <calls> <out.bin>\n");
        return 2;
    }
    const int numDMs = std::atoi(argv[1]), count = std::atoi(argv[2]), calls = std::atoi(argv[3]);
    const float bw = 16e6f, f0 = 1242e6f, period = 0.0005f;
    std::vector<float> bw_i(numDMs, bw), dm_i(numDMs), f0_i(numDMs, f0);
    for (int i = 0; i < numDMs; i++)
        dm_i[i] = 1.0f + 0.5f * i;
    MSOSM_GPU_DM_concurrent msosm(bw_i.data(), dm_i.data(), f0_i.data(), numDMs);
    msosm.initialize_uint16(4096, count);
    const unsigned long process_len = (unsigned long)count * msosm.M_common;

    SimulatedComplexSignal sim(bw, 12.0f, f0, period, "uint16");
    sim.seed = 17;
    sim.generate_pulsar_signal(process_len * calls / sim.Np + 1, true, -3.0f);

    SeriesFileWriter writer(msosm, argv[4]);
    for (int c = 0; c < calls; c++) {
        msosm.filter_block_uint16(sim.signal_u16 + (size_t)c * process_len);
        writer.push();
    }
    std::printf("bytes %llu\n", writer.close());
    return 0;
}
