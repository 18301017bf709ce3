// ref_gpu_runner.cpp -- drives the reference's own GPU classes (cuFFT plus its
// SIMT kernels, compiled from the reference sources for sm_100a) on a B200.
// Test and baseline infrastructure: the GPU parity tests compare this
// library's output with what it writes, and the benchmark times it as "the
// reference path on the same GPU".  Run as a separate process: the
// reference's destructors call cudaDeviceReset.
//
// Inputs are raw uint16_pair files; outputs are record files (see
// ref_golden.cpp).  Every mode refuses trials with Nd == 0: the reference
// leaves delay_points uninitialised there (msosm_prepare.cpp:110-163) and its
// scatter kernel would then index out of bounds.
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <malloc.h>
#include <string>
#include <vector>

#include "msosm_gpu_batch.h"
#include "msosm_gpu_concurrent.h"
#include "osm_gpu_batch.h"
#include "fold_gpu.h"

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
void rec_f64(const char *name, double v) { rec(name, "f8", &v, 1, 8); }

bool read_u16(const char *path, std::vector<uint16_pair> &v, size_t need)
{
    FILE *f = std::fopen(path, "rb");
    if (!f)
        return false;
    v.resize(need);
    size_t got = std::fread(v.data(), sizeof(uint16_pair), need, f);
    std::fclose(f);
    return got == need;
}

bool nd_ok(float bw, float dm, float f0)
{
    Prepare_MSOSM p(bw, dm, f0);
    return dm > 0 && p.Nd >= 1;
}

int usage()
{
    std::fprintf(stderr,
                 "ref_gpu_runner concurrent <fftpoint> <count> <ncalls> <bw> <f0> <in.u16> <out> <dm...>\n"
                 "ref_gpu_runner batch <fftpoint> <count> <ncalls> <bw> <dm> <f0> <in.u16> <out>\n"
                 "ref_gpu_runner osm <fftpoint> <count> <ncalls> <bw> <dm> <f0> <in.u16> <out>\n"
                 "ref_gpu_runner fold2 <fftpoint> <count> <ncalls> <bw> <dm> <f0> <period> <time_bin>"
                 " <a.u16> <b.u16> <out>\n"
                 "ref_gpu_runner time <fftpoint> <count> <ncalls> <repeat> <with_output 0|1> <bw> <f0>"
                 " <in.u16> <out> <dm...>\n"
                 "ref_gpu_runner time1 <batch|osm> <fftpoint> <count> <ncalls> <repeat> <bw> <dm> <f0> <in.u16>"
                 " <out> <write_series 0|1>\n");
    return 2;
}

} // namespace

int main(int argc, char **argv)
{
    if (argc < 2)
        return usage();
    const std::string mode = argv[1];
    if (mode == "concurrent" && argc >= 10) {
        // MSOSM_GPU_DM_concurrent as the reference drivers use it
        // (test_processing_speed_msosm_batch32_dm0to100.cpp:213-293), compute_only
        unsigned long fftpoint = std::strtoul(argv[2], nullptr, 10);
        int count = std::atoi(argv[3]), ncalls = std::atoi(argv[4]);
        float bw = std::strtof(argv[5], nullptr), f0 = std::strtof(argv[6], nullptr);
        int n = argc - 9;
        std::vector<float> bws(n, bw), f0s(n, f0), dms(n);
        for (int i = 0; i < n; i++) {
            dms[i] = std::strtof(argv[9 + i], nullptr);
            if (!nd_ok(bw, dms[i], f0))
                return 5;
        }
        auto *m = new MSOSM_GPU_DM_concurrent(bws.data(), dms.data(), f0s.data(), n);
        m->initialize_uint16(fftpoint, count, 0, true);
        const size_t blk = (size_t)m->count * m->M_common;
        std::vector<uint16_pair> in;
        if (!read_u16(argv[7], in, blk * ncalls))
            return 4;
        g_out = std::fopen(argv[8], "wb");
        rec_u64("M", m->M_common);
        rec_u64("count", (uint64_t)m->count);
        std::vector<Complex> out(blk * n + 1), all;
        for (int c = 0; c < ncalls; c++) {
            m->filter_block_uint16(in.data() + c * blk);
            m->get_output(out.data());
            m->synchronize();
            all.insert(all.end(), out.begin(), out.end() - 1);
        }
        rec("out", "f4", all.data(), 2 * all.size(), 4);
        std::fclose(g_out);
        std::fflush(stdout);
        std::_Exit(0);  // skip the destructor's cudaDeviceReset
    }
    if ((mode == "batch" || mode == "osm") && argc == 10) {
        unsigned long fftpoint = std::strtoul(argv[2], nullptr, 10);
        int count = std::atoi(argv[3]), ncalls = std::atoi(argv[4]);
        float bw = std::strtof(argv[5], nullptr), dm = std::strtof(argv[6], nullptr),
              f0 = std::strtof(argv[7], nullptr);
        if (!nd_ok(bw, dm, f0))
            return 5;
        std::vector<Complex> all;
        unsigned long M = 0;
        size_t blk = 0;
        std::vector<uint16_pair> in;
        if (mode == "batch") {
            MSOSM_GPU_BATCH m(bw, dm, f0);
            m.initialize_uint16(fftpoint, count);
            M = m.M;
            blk = (size_t)count * M;
            if (!read_u16(argv[8], in, blk * ncalls))
                return 4;
            std::vector<Complex> out(blk);
            for (int c = 0; c < ncalls; c++) {
                m.filter_block_uint16(in.data() + c * blk);
                m.get_output(out.data());
                all.insert(all.end(), out.begin(), out.end());
            }
        } else {
            OSM_GPU_BATCH m(bw, dm, f0);
            m.initialize_uint16(fftpoint, count, false);
            M = m.M;
            blk = (size_t)count * M;
            if (!read_u16(argv[8], in, blk * ncalls))
                return 4;
            std::vector<Complex> out(blk);
            for (int c = 0; c < ncalls; c++) {
                m.filter_block_uint16(in.data() + c * blk);
                m.get_output(out.data());
                all.insert(all.end(), out.begin(), out.end());
            }
        }
        g_out = std::fopen(argv[9], "wb");
        rec_u64("M", M);
        rec_u64("count", (uint64_t)count);
        rec("out", "f4", all.data(), 2 * all.size(), 4);
        std::fclose(g_out);
        return 0;
    }
    if (mode == "fold2" && argc == 13) {
        // msosm_psrdada.cpp:105-142: two MSOSM_GPU_BATCH (one per pol),
        // Fold_GPU::calculate_intensity + fold_data per block, fold_data_bins
        unsigned long fftpoint = std::strtoul(argv[2], nullptr, 10);
        int count = std::atoi(argv[3]), ncalls = std::atoi(argv[4]);
        float bw = std::strtof(argv[5], nullptr), dm = std::strtof(argv[6], nullptr),
              f0 = std::strtof(argv[7], nullptr), period = std::strtof(argv[8], nullptr);
        long tb = std::strtol(argv[9], nullptr, 10);
        if (!nd_ok(bw, dm, f0))
            return 5;
        // Fold_GPU allocates folded_data_raw / tmp_fold / fold_count with new[]
        // and accumulates into them without clearing (fold_gpu.cpp:15-18):
        // serve every allocation from fresh zeroed pages so its sums start at 0.
        mallopt(M_MMAP_THRESHOLD, 0);
        MSOSM_GPU_BATCH a(bw, dm, f0), b(bw, dm, f0);
        a.initialize_uint16(fftpoint, count);
        b.initialize_uint16(fftpoint, count);
        const size_t blk = (size_t)count * a.M;
        std::vector<uint16_pair> ina, inb;
        if (!read_u16(argv[10], ina, blk * ncalls) || !read_u16(argv[11], inb, blk * ncalls))
            return 4;
        Fold_GPU fold(period, bw, blk, "/dev/null", tb < 0 ? (unsigned long)-1 : (unsigned long)tb);
        fold.discard_samples(a.Nd);
        for (int c = 0; c < ncalls; c++) {
            a.filter_block_uint16(ina.data() + c * blk);
            b.filter_block_uint16(inb.data() + c * blk);
            fold.calculate_intensity<MSOSM_GPU_BATCH>(&a, &b);
            fold.fold_data();
        }
        fold.fold_data_bins();
        g_out = std::fopen(argv[12], "wb");
        rec_u64("M", a.M);
        rec_u64("Nd", a.Nd);
        rec_u64("period_samples", fold.period_samples);
        rec_u64("time_bin", fold.time_bin);
        rec("folded", "f4", fold.folded_data, fold.time_bin, 4);
        std::fclose(g_out);
        return 0;
    }
    if (mode == "time" && argc >= 12) {
        // the reference's own timing methodology
        // (test_processing_speed_msosm_batch32_dm0to100.cpp:259-302): input
        // registered with cudaHostRegister, std::chrono around the
        // filter_block_uint16 (+ get_output) loop and synchronize()
        unsigned long fftpoint = std::strtoul(argv[2], nullptr, 10);
        int count = std::atoi(argv[3]), ncalls = std::atoi(argv[4]), repeat = std::atoi(argv[5]);
        int with_output = std::atoi(argv[6]);
        float bw = std::strtof(argv[7], nullptr), f0 = std::strtof(argv[8], nullptr);
        int n = argc - 11;
        std::vector<float> bws(n, bw), f0s(n, f0), dms(n);
        for (int i = 0; i < n; i++) {
            dms[i] = std::strtof(argv[11 + i], nullptr);
            if (!nd_ok(bw, dms[i], f0))
                return 5;
        }
        auto *m = new MSOSM_GPU_DM_concurrent(bws.data(), dms.data(), f0s.data(), n);
        m->initialize_uint16(fftpoint, count, 0, true);
        const size_t blk = (size_t)m->count * m->M_common;
        std::vector<uint16_pair> in;
        if (!read_u16(argv[9], in, blk * ncalls))
            return 4;
        if (cudaHostRegister(in.data(), in.size() * sizeof(uint16_pair), cudaHostRegisterDefault) != cudaSuccess)
            return 6;
        std::vector<Complex> out;
        if (with_output) {
            out.resize(blk * n + 1);
            if (cudaHostRegister(out.data(), out.size() * sizeof(Complex), cudaHostRegisterDefault) != cudaSuccess)
                return 6;
        }
        std::vector<double> ms;
        for (int r = 0; r < repeat + 1; r++) {  // first run is warm-up
            auto t0 = std::chrono::high_resolution_clock::now();
            for (int c = 0; c < ncalls; c++) {
                m->filter_block_uint16(in.data() + c * blk);
                if (with_output)
                    m->get_output(out.data());
            }
            m->synchronize();
            auto t1 = std::chrono::high_resolution_clock::now();
            if (r > 0)
                ms.push_back(std::chrono::duration<double, std::milli>(t1 - t0).count());
        }
        g_out = std::fopen(argv[10], "wb");
        rec_u64("M", m->M_common);
        rec_u64("count", (uint64_t)m->count);
        rec("ms", "f8", ms.data(), ms.size(), 8);
        std::fclose(g_out);
        std::_Exit(0);
    }
    if (mode == "time1" && argc == 13) {
        // one DM through the single-trial classes, timed the way the
        // reference's single-DM speed tests time them
        // (test_processing_speed_msosm.cpp:198-221): input and output
        // registered with cudaHostRegister, std::chrono around the
        // filter_block_uint16 + get_output loop and a final synchronize.
        // MSOSM_GPU_BATCH / OSM_GPU_BATCH copy with plain cudaMemcpy
        // (msosm_gpu_batch.cpp:75-99, osm_gpu_batch.cpp:94-128).  The series
        // of the first (warm-up) run is written out for the parity check.
        const std::string kind = argv[2];
        unsigned long fftpoint = std::strtoul(argv[3], nullptr, 10);
        int count = std::atoi(argv[4]), ncalls = std::atoi(argv[5]), repeat = std::atoi(argv[6]);
        float bw = std::strtof(argv[7], nullptr), dm = std::strtof(argv[8], nullptr),
              f0 = std::strtof(argv[9], nullptr);
        if (!nd_ok(bw, dm, f0) || (kind != "batch" && kind != "osm"))
            return 5;
        MSOSM_GPU_BATCH *ms = nullptr;
        OSM_GPU_BATCH *os = nullptr;
        unsigned long M = 0;
        if (kind == "batch") {
            ms = new MSOSM_GPU_BATCH(bw, dm, f0);
            ms->initialize_uint16(fftpoint, count);
            M = ms->M;
        } else {
            os = new OSM_GPU_BATCH(bw, dm, f0);
            os->initialize_uint16(fftpoint, count, false);
            M = os->M;
        }
        const size_t blk = (size_t)count * M;
        std::vector<uint16_pair> in;
        if (!read_u16(argv[10], in, blk * ncalls))
            return 4;
        // the first run's series (the stream from its start) is the one
        // written out; later runs continue the stream and write elsewhere
        std::vector<Complex> out(blk * ncalls), again(blk * ncalls);
        if (cudaHostRegister(in.data(), in.size() * sizeof(uint16_pair), cudaHostRegisterDefault) != cudaSuccess ||
            cudaHostRegister(out.data(), out.size() * sizeof(Complex), cudaHostRegisterDefault) != cudaSuccess ||
            cudaHostRegister(again.data(), again.size() * sizeof(Complex), cudaHostRegisterDefault) != cudaSuccess)
            return 6;
        std::vector<double> ms_v;
        for (int r = 0; r < repeat + 1; r++) {  // first run is warm-up
            Complex *dst = r == 0 ? out.data() : again.data();
            auto t0 = std::chrono::high_resolution_clock::now();
            for (int c = 0; c < ncalls; c++) {
                if (ms) {
                    ms->filter_block_uint16(in.data() + c * blk);
                    ms->get_output(dst + c * blk);
                } else {
                    os->filter_block_uint16(in.data() + c * blk);
                    os->get_output(dst + c * blk);
                }
            }
            cudaDeviceSynchronize();
            auto t1 = std::chrono::high_resolution_clock::now();
            if (r > 0)
                ms_v.push_back(std::chrono::duration<double, std::milli>(t1 - t0).count());
        }
        g_out = std::fopen(argv[11], "wb");
        rec_u64("M", M);
        rec_u64("count", (uint64_t)count);
        rec("ms", "f8", ms_v.data(), ms_v.size(), 8);
        if (std::atoi(argv[12]))
            rec("out", "f4", out.data(), 2 * out.size(), 4);
        std::fclose(g_out);
        std::fflush(stdout);
        std::_Exit(0);
    }
    return usage();
}
