// ref_golden.cpp -- drives the reference's own HOST code (filter design,
// segmentation, Fold_GPU::fold_data, SimulatedComplexSignal) compiled from the
// reference sources in place, and dumps what it computes.  Test
// infrastructure: its outputs become the committed golden fixtures under
// tests/golden/ (tests/golden/make_golden.py runs it).  Runs on a CPU: none of
// the calls below launches a kernel.
//
// Output: a record file; each record is
//   char name[32]; char dtype[8]; uint64 count; count elements of dtype.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <malloc.h>
#include <string>
#include <vector>

#include "prepare.h"
#include "prepare_concurrent.h"
#include "fold_gpu.h"
#include "simulated_complex_signal.h"
#include "psrdada.h"

namespace {

FILE *g_out = nullptr;

void rec(const char *name, const char *dtype, const void *data, uint64_t count, size_t elem)
{
    char n[32] = {0}, d[8] = {0};
    std::strncpy(n, name, 31);
    std::strncpy(d, dtype, 7);
    std::fwrite(n, 1, 32, g_out);
    std::fwrite(d, 1, 8, g_out);
    std::fwrite(&count, 8, 1, g_out);
    if (count)
        std::fwrite(data, elem, count, g_out);
}

void rec_u64(const char *name, uint64_t v) { rec(name, "u8", &v, 1, 8); }

int usage()
{
    std::fprintf(stderr,
                 "ref_golden msosm <bw> <dm> <f0> <fftpoint> <out>\n"
                 "ref_golden concurrent <bw> <f0> <fftpoint> <out> <dm...>\n"
                 "ref_golden osm <bw> <dm> <f0> <fftpoint> <out>\n"
                 "ref_golden fold <period> <fs> <size> <time_bin|-1> <Nd|-1> <nchunks> <in.f32> <out>\n"
                 "ref_golden simulate <bw> <dm> <f0> <period> <repeat> <out>\n"
                 "ref_golden dada <file> <n> <reads> <out>\n");
    return 2;
}

} // namespace

int main(int argc, char **argv)
{
    // Fold_GPU allocates folded_data_raw / tmp_fold / fold_count with new[]
    // and accumulates into them without clearing (fold_gpu.cpp:15-18): serve
    // every allocation from fresh zeroed pages so its sums start at zero.
    mallopt(M_MMAP_THRESHOLD, 0);
    if (argc < 2)
        return usage();
    std::string mode = argv[1];
    if (mode == "msosm" && argc == 7) {
        // MSOSM_GPU_BATCH::initialize_uint16 host part (msosm_gpu_batch.cpp:12-31)
        float bw = std::strtof(argv[2], nullptr), dm = std::strtof(argv[3], nullptr),
              f0 = std::strtof(argv[4], nullptr);
        unsigned long fftpoint = std::strtoul(argv[5], nullptr, 10);
        g_out = std::fopen(argv[6], "wb");
        Prepare_MSOSM p(bw, dm, f0);
        p.calculate_min_order();
        if (fftpoint != 0) {
            p.M = fftpoint / 2;
            if (p.M < p.M_min)
                p.M = p.M_min;
        }
        p.segmentation();
        p.generate_dedisp_params();
        rec_u64("Nd", p.Nd);
        rec_u64("M_min", p.M_min);
        rec_u64("M", p.M);
        rec_u64("delaycount", (uint64_t)p.delaycount);
        rec("delay_points", "i4", p.delay_points, 2 * p.M, 4);
        rec("H", "f4", p.dedisp_params, 4 * p.M, 4);
    } else if (mode == "concurrent" && argc >= 7) {
        // MSOSM_GPU_DM_concurrent::initialize_uint16 host part
        // (msosm_gpu_dm_concurrent.cpp:28-38,81-103)
        float bw = std::strtof(argv[2], nullptr), f0 = std::strtof(argv[3], nullptr);
        unsigned long fftpoint = std::strtoul(argv[4], nullptr, 10);
        g_out = std::fopen(argv[5], "wb");
        int n = argc - 6;
        std::vector<float> bws(n, bw), f0s(n, f0), dms(n);
        for (int i = 0; i < n; i++)
            dms[i] = std::strtof(argv[6 + i], nullptr);
        Prepare_MSOSM_DM_concurrent p(bws.data(), dms.data(), f0s.data(), n);
        p.calculate_min_order();
        if (fftpoint != 0) {
            p.M_common = fftpoint / 2;
            if (p.M_common < p.M_common_min)
                p.M_common = p.M_common_min;
        }
        rec_u64("M_common", p.M_common);
        rec_u64("M_common_min", p.M_common_min);
        std::vector<uint64_t> nd(n), mmin(n), dc(n);
        std::vector<int32_t> dp;
        std::vector<float> H;
        for (int i = 0; i < n; i++) {
            p.segmentation(i);
            p.generate_dedisp_params(i);
            nd[i] = p.Nd[i];
            mmin[i] = p.M_min[i];
            dc[i] = (uint64_t)p.delaycount[i];
            dp.insert(dp.end(), p.delay_points[i], p.delay_points[i] + 2 * p.M_common);
            float *h = reinterpret_cast<float *>(p.dedisp_params[i]);
            H.insert(H.end(), h, h + 4 * p.M_common);
        }
        rec("Nd", "u8", nd.data(), n, 8);
        rec("M_min", "u8", mmin.data(), n, 8);
        rec("delaycount", "u8", dc.data(), n, 8);
        rec("delay_points", "i4", dp.data(), dp.size(), 4);
        rec("H", "f4", H.data(), H.size(), 4);
    } else if (mode == "osm" && argc == 7) {
        // OSM_GPU_BATCH::initialize_uint16 host part (osm_gpu_batch.cpp:30-43)
        float bw = std::strtof(argv[2], nullptr), dm = std::strtof(argv[3], nullptr),
              f0 = std::strtof(argv[4], nullptr);
        unsigned long fftpoint = std::strtoul(argv[5], nullptr, 10);
        g_out = std::fopen(argv[6], "wb");
        Prepare_OSM p(bw, dm, f0);
        p.calculate_min_order();
        if (fftpoint != 0) {
            p.M = fftpoint / 2;
            if (p.M < p.M_min)
                p.M = p.M_min;
        }
        p.generate_dedisp_params();
        rec_u64("Nd", p.Nd);
        rec_u64("M_min", p.M_min);
        rec_u64("M", p.M);
        rec("H", "f4", p.dedisp_params, 4 * p.M, 4);
    } else if (mode == "fold" && argc == 10) {
        // Fold_GPU fed chunk by chunk through its public total_intensity
        // buffer (fold_gpu.cpp:48-194), as msosm_psrdada.cpp:136-142 does.
        float period = std::strtof(argv[2], nullptr), fs = std::strtof(argv[3], nullptr);
        unsigned long size = std::strtoul(argv[4], nullptr, 10);
        long tb = std::strtol(argv[5], nullptr, 10);
        long nd = std::strtol(argv[6], nullptr, 10);
        int nchunks = std::atoi(argv[7]);
        FILE *in = std::fopen(argv[8], "rb");
        g_out = std::fopen(argv[9], "wb");
        if (!in || !g_out)
            return 3;
        Fold_GPU fold(period, fs, size, "/dev/null", tb < 0 ? (unsigned long)-1 : (unsigned long)tb);
        if (nd >= 0)
            fold.discard_samples((unsigned long)nd);
        for (int c = 0; c < nchunks; c++) {
            if (std::fread(fold.total_intensity, sizeof(float), size, in) != size)
                return 4;
            fold.fold_data();
        }
        fold.fold_data_bins();
        rec_u64("period_samples", fold.period_samples);
        rec_u64("time_bin", fold.time_bin);
        rec("folded", "f4", fold.folded_data, fold.time_bin, 4);
        std::fclose(in);
    } else if (mode == "simulate" && argc == 8) {
        // SimulatedComplexSignal::generate_pulsar_signal without noise,
        // unpinned (simulated_complex_signal.cpp:40-236)
        float bw = std::strtof(argv[2], nullptr), dm = std::strtof(argv[3], nullptr),
              f0 = std::strtof(argv[4], nullptr), period = std::strtof(argv[5], nullptr);
        unsigned long repeat = std::strtoul(argv[6], nullptr, 10);
        g_out = std::fopen(argv[7], "wb");
        SimulatedComplexSignal s(bw, dm, f0, period, "uint16");
        s.generate_pulsar_signal(repeat, false, 0, false);
        rec_u64("Np", s.Np);
        rec_u64("Nd", s.Nd);
        rec("signal", "f4", s.signal, 2 * s.signal_size, 4);
        rec("signal_u16", "u2", s.signal_u16, 2 * s.signal_size, 2);
    } else if (mode == "dada" && argc == 6) {
        // PSRDADA::PSRDADA + initBuffer + readSamples (psrdada/psrdada.cpp:3-94)
        unsigned long n = std::strtoul(argv[3], nullptr, 10);
        int reads = std::atoi(argv[4]);
        g_out = std::fopen(argv[5], "wb");
        PSRDADA file(argv[2]);
        file.initBuffer(n);
        float f[2] = {file.bw, file.fc};
        int32_t i[4] = {file.nbit, file.nchan, file.ndim, file.npol};
        rec("bw_fc", "f4", f, 2, 4);
        rec("nbit_nchan_ndim_npol", "i4", i, 4, 4);
        rec_u64("filesize", file.filesize);
        rec_u64("readCount", file.readCount);
        rec_u64("frameCount", (uint64_t)file.frameCount);
        std::vector<uint16_pair> p1, p2;
        for (int r = 0; r < reads; r++) {
            file.readSamples();
            p1.insert(p1.end(), file.pol1_in, file.pol1_in + n);
            p2.insert(p2.end(), file.pol2_in, file.pol2_in + n);
        }
        rec("pol1", "u2", p1.data(), 2 * p1.size(), 2);
        rec("pol2", "u2", p2.data(), 2 * p2.size(), 2);
    } else {
        return usage();
    }
    std::fclose(g_out);
    return 0;
}
