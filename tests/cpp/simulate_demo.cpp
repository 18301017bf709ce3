// simulate_demo.cpp -- the reference drivers' use of the simulator
// (check_msosm.cpp:100-110: SimulatedComplexSignal in "uint16" mode, then
// generate_pulsar_signal(repeat, add_noise, SNR)) and of AWGN, written
// against the drop-in header.  Writes the complex signal, its uint16 pairs
// and n AWGN(SNR, n) samples to <out>, in that order.
//
//   simulate_demo <bw> <dm> <f0> <period> <repeat> <add_noise> <snr_db> <seed> <n_awgn> <out>
#include <cstdio>
#include <cstdlib>

#include "msosm_gpu_b200.hpp"

using namespace msosm_b200;

int main(int argc, char **argv)
{
    if (argc != 11) {
        std::fprintf(stderr, "usage: simulate_demo <bw> <dm> <f0> <period> <repeat> <add_noise> <snr_db> <seed> "
                             "<n_awgn> <out>\n");
        return 2;
    }
    const float bw = std::strtof(argv[1], nullptr), dm = std::strtof(argv[2], nullptr),
                f0 = std::strtof(argv[3], nullptr), period = std::strtof(argv[4], nullptr);
    const unsigned long repeat = std::strtoul(argv[5], nullptr, 10);
    const bool add_noise = std::atoi(argv[6]) != 0;
    const float snr = std::strtof(argv[7], nullptr);
    const unsigned long long seed = std::strtoull(argv[8], nullptr, 10);
    const unsigned long n_awgn = std::strtoul(argv[9], nullptr, 10);

    SimulatedComplexSignal *simulated_signal = new SimulatedComplexSignal(bw, dm, f0, period, "uint16");
    simulated_signal->seed = seed;
    simulated_signal->generate_pulsar_signal(repeat, add_noise, snr);
    std::printf("Np %lu Nd %lu range %lu signal_size %lu power %.6f dB\n", simulated_signal->Np,
                simulated_signal->Nd, simulated_signal->range, simulated_signal->signal_size,
                simulated_signal->signal_power);

    AWGN g(snr, n_awgn);
    g.seed = seed;
    Complex *noise = g.generateNoiseSamples();

    std::FILE *f = std::fopen(argv[10], "wb");
    if (!f)
        return 3;
    std::fwrite(simulated_signal->signal, sizeof(Complex), simulated_signal->signal_size, f);
    std::fwrite(simulated_signal->signal_u16, sizeof(uint16_pair), simulated_signal->signal_size, f);
    std::fwrite(noise, sizeof(Complex), n_awgn, f);
    std::fclose(f);
    g.deallocate();
    delete simulated_signal;
    return 0;
}
