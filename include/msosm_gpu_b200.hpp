// msosm_gpu_b200.hpp -- header-only C++ drop-in for the reference's host API.
//
// The classes below carry the names, constructor/method signatures and
// public fields of the reference classes in dedispersion/include/*.h
// (msosm_gpu_batch.h, msosm_gpu_concurrent.h, msosm_gpu_batch_stream.h,
// osm_gpu_batch.h, osm_gpu_concurrent.h, prepare*.h) and call the C ABI of
// libmsosm_b200.so (msosm_b200.h).  A program written against the
// reference builds against this header by swapping its includes and linking
// -lmsosm_b200; it needs neither FFTW nor cuFFT.
//
// Differences a caller can observe:
//  * errors print a message and exit(1) like the reference's CUDA_CHECK
//    (gpu/include/gpu_common.cuh:41-61); define MSOSM_B200_THROW before the
//    include to get std::runtime_error instead;
//  * dedisp_params is msosm_complex* (same layout as fftwf_complex);
//  * reset_device() and the destructors release this object's resources
//    only (the reference calls cudaDeviceReset, which ends every allocation
//    of the process);
//  * get_output() waits for the copy, so the wait_for_cpu / wait_for_threads
//    handshake of the reference (a busy-wait on a plain bool,
//    msosm_gpu_dm_concurrent.cpp:156-160) is kept as fields but never spins;
//  * trials with DM 0 get all block delays 0 (undefined in the reference).
#pragma once

#include <algorithm>
#include <cstdio>
#include <ctime>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

#include "msosm_b200.h"

namespace msosm_b200 {

using Complex = msosm_complex;
using uint16_pair = msosm_uint16_pair;

// Not in the reference: MS-OSM objects initialised after use_tensor_cores(true)
// run their inverse transforms on the tensor cores (MSOSM_FLAG_TENSOR_F16: f16
// operands, f32 accumulation, FFT sizes 4096 and 8192; series error ~5e-4
// relative RMS, folded profiles ~3e-5).  Off by default.
inline unsigned int &extra_flags()
{
    static unsigned int f = 0;
    return f;
}
inline void use_tensor_cores(bool on, bool bf16 = false)
{
    extra_flags() = on ? (bf16 ? MSOSM_FLAG_TENSOR_BF16 : MSOSM_FLAG_TENSOR_F16) : 0u;
}

inline void check(msosm_status s, const char *what)
{
    if (s == MSOSM_OK)
        return;
    std::string msg = std::string(what) + ": " + msosm_last_error();
#ifdef MSOSM_B200_THROW
    throw std::runtime_error(msg);
#else
    std::fprintf(stderr, "msosm error %d: %s\n", s, msg.c_str());
    std::exit(1);
#endif
}

// ---------------------------------------------------------------------------
// filter design (dedispersion/include/prepare.h:7-49, :101-134)
// ---------------------------------------------------------------------------

class Prepare_MSOSM {
public:
    explicit Prepare_MSOSM(float bw = 0, float dm = 0, float f0 = 0) : bw_(bw), dm_(dm), f0_(f0)
    {
        if (bw > 0 && f0 > 0)
            check(msosm_prepare_nd(bw, dm, f0, &Nd), "msosm_prepare_nd");
    }
    void calculate_min_order()
    {
        check(msosm_prepare_min_order_msosm(Nd, &M), "msosm_prepare_min_order_msosm");
        M_min = M;
    }
    void override_order(unsigned long order) { M = order; }
    void segmentation()
    {
        dp_.assign(2 * M, 0);
        check(msosm_prepare_segmentation(bw_, dm_, f0_, M, &delaycount, dp_.data()), "segmentation");
        delay_points = dp_.data();
    }
    void generate_dedisp_params()
    {
        H_.assign(2 * M, Complex{0.f, 0.f});
        check(msosm_prepare_dedisp_params(bw_, dm_, f0_, M, H_.data()), "generate_dedisp_params");
        dedisp_params = H_.data();
    }

    unsigned long M = 0, M_min = 0;
    int delaycount = 0;
    Complex *dedisp_params = nullptr;
    int *delay_points = nullptr;
    unsigned long Nd = 0;

protected:
    float bw_, dm_, f0_;
    std::vector<int> dp_;
    std::vector<Complex> H_;
};

namespace detail {

// One msosm_dedisp handle plus the reference-shaped views of its state.
class Handle {
public:
    Handle() = default;
    Handle(const Handle &) = delete;
    Handle &operator=(const Handle &) = delete;
    ~Handle() { reset(); }
    void create(const float *bw, const float *dm, const float *f0, int n, unsigned long fftpoint, int count,
                unsigned long input_size, unsigned int flags)
    {
        reset();
        check(msosm_dedisp_create(bw, dm, f0, n, fftpoint, count, input_size, flags, &h), "msosm_dedisp_create");
        check(msosm_dedisp_get_info(h, &info), "msosm_dedisp_get_info");
        n_ = n;
        Nd.resize(n);
        delaycount.resize(n);
        check(msosm_dedisp_get_nd(h, Nd.data()), "msosm_dedisp_get_nd");
        check(msosm_dedisp_get_delaycount(h, delaycount.data()), "msosm_dedisp_get_delaycount");
        dp.assign((size_t)n * info.fftpoint, 0);
        H.assign((size_t)n * info.fftpoint, Complex{0.f, 0.f});
        for (int i = 0; i < n; ++i) {
            check(msosm_dedisp_get_delay_points(h, i, dp.data() + (size_t)i * info.fftpoint), "delay_points");
            check(msosm_dedisp_get_dedisp_params(h, i, H.data() + (size_t)i * info.fftpoint), "dedisp_params");
        }
    }
    void reset()
    {
        if (h)
            msosm_dedisp_destroy(h);
        h = nullptr;
    }
    size_t block() const { return (size_t)info.count * info.M; }
    Complex *device_output() const
    {
        Complex *p = nullptr;
        check(msosm_dedisp_output_device_ptr(h, &p), "msosm_dedisp_output_device_ptr");
        return p;
    }

    msosm_dedisp *h = nullptr;
    msosm_dedisp_info info{};
    int n_ = 0;
    std::vector<unsigned long> Nd;
    std::vector<int> delaycount;
    std::vector<int> dp;
    std::vector<Complex> H;
};

}  // namespace detail

// ---------------------------------------------------------------------------
// single DM (dedispersion/include/msosm_gpu_batch.h:7-41)
// ---------------------------------------------------------------------------

class MSOSM_GPU_BATCH : public Prepare_MSOSM {
public:
    explicit MSOSM_GPU_BATCH(float bw = 0, float dm = 0, float f0 = 0) : Prepare_MSOSM(bw, dm, f0) {}
    void get_device_info() { std::printf("CUDA devices: %d\n", msosm_device_count()); }
    void initialize_uint16(unsigned long fftpoint = 0, int count = 1)
    {
        h_.create(&bw_, &dm_, &f0_, 1, fftpoint, count, 0, extra_flags());
        M = h_.info.M;
        M_min = h_.info.M_min;
        this->count = h_.info.count;
        delaycount = h_.delaycount[0];
        delay_points = h_.dp.data();
        dedisp_params = h_.H.data();
        output_buffer_d = h_.device_output();
    }
    void filter_block_uint16(uint16_pair *input)
    {
        check(msosm_dedisp_filter_block_uint16(h_.h, input), "filter_block_uint16");
    }
    void get_output(Complex *output)
    {
        // the handle's buffer ends with one extra element; copy count*M
        out_.resize(h_.block() + 1);
        check(msosm_dedisp_get_output_c64(h_.h, out_.data()), "get_output");
        std::copy(out_.begin(), out_.end() - 1, output);
    }

    int count = 0;
    Complex *output_buffer_d = nullptr;
    msosm_dedisp *handle() const { return h_.h; }

protected:
    detail::Handle h_;
    std::vector<Complex> out_;
};

// classical overlap-save (dedispersion/include/osm_gpu_batch.h:7-37)
class OSM_GPU_BATCH : public MSOSM_GPU_BATCH {
public:
    explicit OSM_GPU_BATCH(float bw = 0, float dm = 0, float f0 = 0) : MSOSM_GPU_BATCH(bw, dm, f0) {}
    void initialize_uint16(unsigned long fftpoint = 0, int count = 1, bool streaming = false)
    {
        (void)streaming;
        h_.create(&bw_, &dm_, &f0_, 1, fftpoint, count, 0, MSOSM_FLAG_OSM);
        M = h_.info.M;
        M_min = h_.info.M_min;
        this->count = h_.info.count;
        dedisp_params = h_.H.data();
        output_buffer_d = h_.device_output();
        total_memory = h_.info.device_bytes;
    }
    unsigned long total_memory = 0;
};

// ---------------------------------------------------------------------------
// many DMs over one input (dedispersion/include/msosm_gpu_concurrent.h:15-64)
// ---------------------------------------------------------------------------

class MSOSM_GPU_DM_concurrent {
public:
    MSOSM_GPU_DM_concurrent(float *bw, float *dm, float *f0, int numDMs)
        : numDMs(numDMs), bw_(bw, bw + numDMs), dm_(dm, dm + numDMs), f0_(f0, f0 + numDMs)
    {
    }
    virtual ~MSOSM_GPU_DM_concurrent() = default;
    void get_device_info() { std::printf("CUDA devices: %d\n", msosm_device_count()); }
    void initialize_uint16(unsigned long fftpoint, int count = 1, unsigned long input_size = 0,
                           bool compute_only = false)
    {
        create(fftpoint, count, input_size, extra_flags());
        this->compute_only = compute_only;
    }
    void initialize_threads_flag(int thread_num) { wait_for_threads.assign(thread_num, false); }
    void filter_block_uint16(uint16_pair *input)
    {
        check(msosm_dedisp_filter_block_uint16(h_.h, input), "filter_block_uint16");
    }
    // numDMs*count*M + 1 elements, [dm][count*M] then a trailing zero
    void get_output(Complex *output) { check(msosm_dedisp_get_output_c64(h_.h, output), "get_output"); }
    void get_output(uint16_pair *output)
    {
        check(msosm_dedisp_get_output_uint16(h_.h, output), "get_output");
    }
    void get_output_thread(uint16_pair *output, int thread_id)
    {
        (void)thread_id;
        get_output(output);
    }
    void synchronize() { check(msosm_dedisp_synchronize(h_.h), "synchronize"); }
    void reset_device() { h_.reset(); }
    msosm_dedisp *handle() const { return h_.h; }

    int count = 0;
    bool wait_for_cpu = false;
    std::vector<bool> wait_for_threads;
    unsigned long M_common = 0, M_common_min = 0;
    std::vector<unsigned long> Nd;
    std::vector<int> delaycount;
    int numDMs;
    // per-trial views (Prepare_MSOSM_DM_concurrent::delay_points / dedisp_params)
    int *delay_points_of(int i) { return h_.dp.data() + (size_t)i * h_.info.fftpoint; }
    Complex *dedisp_params_of(int i) { return h_.H.data() + (size_t)i * h_.info.fftpoint; }

protected:
    void create(unsigned long fftpoint, int count, unsigned long input_size, unsigned int flags)
    {
        h_.create(bw_.data(), dm_.data(), f0_.data(), numDMs, fftpoint, count, input_size, flags);
        this->count = h_.info.count;
        M_common = h_.info.M;
        M_common_min = h_.info.M_min;
        Nd = h_.Nd;
        delaycount = h_.delaycount;
    }
    bool compute_only = false;
    std::vector<float> bw_, dm_, f0_;
    detail::Handle h_;
};

// dedispersion/include/osm_gpu_concurrent.h:7-42
class OSM_GPU_DM_concurrent : public MSOSM_GPU_DM_concurrent {
public:
    using MSOSM_GPU_DM_concurrent::MSOSM_GPU_DM_concurrent;
    void initialize_uint16(unsigned long fftpoint = 0, int count = 1, bool compute_only = false)
    {
        create(fftpoint, count, 0, MSOSM_FLAG_OSM);
        this->compute_only = compute_only;
    }
};

// ---------------------------------------------------------------------------
// one DM per output, one input, processed DM by DM
// (dedispersion/include/msosm_gpu_batch.h:43-77)
// ---------------------------------------------------------------------------

class MSOSM_GPU_DM_BATCH_loop {
public:
    MSOSM_GPU_DM_BATCH_loop(float *bw, float *dm, float *f0, int numOutput)
        : numOutput(numOutput), bw_(bw, bw + numOutput), dm_(dm, dm + numOutput), f0_(f0, f0 + numOutput)
    {
    }
    void get_device_info() { std::printf("CUDA devices: %d\n", msosm_device_count()); }
    void initialize_uint16(unsigned long fftpoint, int count = 1)
    {
        h_.create(bw_.data(), dm_.data(), f0_.data(), numOutput, fftpoint, count, 0, extra_flags());
        this->count = h_.info.count;
        M_loop = h_.info.M;
        M_loop_min = h_.info.M_min;
        Nd = h_.Nd;
        delaycount = h_.delaycount;
    }
    // every trial is dedispersed here; filter_block_uint16(out, i) then
    // copies trial i (the reference runs trial i's filter at that point)
    void input_process(uint16_pair *input)
    {
        check(msosm_dedisp_filter_block_uint16(h_.h, input), "input_process");
        all_.resize((size_t)numOutput * h_.block() + 1);
        check(msosm_dedisp_get_output_c64(h_.h, all_.data()), "get_output");
    }
    void filter_block_uint16(Complex **output, int i)
    {
        std::copy(all_.begin() + (size_t)i * h_.block(), all_.begin() + (size_t)(i + 1) * h_.block(), output[i]);
    }
    void synchronize() { check(msosm_dedisp_synchronize(h_.h), "synchronize"); }

    int count = 0;
    int numOutput;
    unsigned long M_loop = 0, M_loop_min = 0;
    std::vector<unsigned long> Nd;
    std::vector<int> delaycount;

private:
    std::vector<float> bw_, dm_, f0_;
    detail::Handle h_;
    std::vector<Complex> all_;
};

// one DM per stream over one input (dedispersion/include/msosm_gpu_batch_stream.h:52-93)
class MSOSM_GPU_DM_BATCH_stream : public MSOSM_GPU_DM_concurrent {
public:
    MSOSM_GPU_DM_BATCH_stream(float *bw, float *dm, float *f0, int numStreams)
        : MSOSM_GPU_DM_concurrent(bw, dm, f0, numStreams), numStreams(numStreams)
    {
    }
    void initialize_uint16(unsigned long fftpoint, int count = 1)
    {
        create(fftpoint, count, 0, extra_flags());
        M_stream = M_common;
        M_stream_min = M_common_min;
    }
    void get_output(Complex **output)
    {
        all_.resize((size_t)numStreams * block() + 1);
        check(msosm_dedisp_get_output_c64(h_.h, all_.data()), "get_output");
        for (int i = 0; i < numStreams; ++i)
            std::copy(all_.begin() + (size_t)i * block(), all_.begin() + (size_t)(i + 1) * block(), output[i]);
    }
    void get_output(uint16_pair **output)
    {
        u_.resize((size_t)numStreams * block() + 1);
        check(msosm_dedisp_get_output_uint16(h_.h, u_.data()), "get_output");
        for (int i = 0; i < numStreams; ++i)
            std::copy(u_.begin() + (size_t)i * block(), u_.begin() + (size_t)(i + 1) * block(), output[i]);
    }
    int numStreams;
    unsigned long M_stream = 0, M_stream_min = 0;

private:
    size_t block() const { return (size_t)count * M_common; }
    std::vector<Complex> all_;
    std::vector<uint16_pair> u_;
};

// ---------------------------------------------------------------------------
// independent single-DM pipelines, one input each
// (dedispersion/include/msosm_gpu_batch_stream.h:14-49)
// ---------------------------------------------------------------------------

class MSOSM_GPU_BATCH_stream {
public:
    MSOSM_GPU_BATCH_stream(float *bw, float *dm, float *f0, int numStreams)
        : numStreams(numStreams), bw_(bw, bw + numStreams), dm_(dm, dm + numStreams), f0_(f0, f0 + numStreams),
          h_(numStreams)
    {
    }
    void get_device_info() { std::printf("CUDA devices: %d\n", msosm_device_count()); }
    // fftpoint[i] per stream (raised to the minimum and written back, as the reference does)
    void initialize_uint16(unsigned long *fftpoint, int count = 1)
    {
        M.resize(numStreams);
        M_min.resize(numStreams);
        Nd.resize(numStreams);
        delaycount.resize(numStreams);
        output_buffer_d.resize(numStreams);
        for (int i = 0; i < numStreams; ++i) {
            h_[i].create(&bw_[i], &dm_[i], &f0_[i], 1, fftpoint[i], count, 0, 0);
            M[i] = h_[i].info.M;
            M_min[i] = h_[i].info.M_min;
            fftpoint[i] = h_[i].info.fftpoint;
            Nd[i] = h_[i].Nd[0];
            delaycount[i] = h_[i].delaycount[0];
            output_buffer_d[i] = h_[i].device_output();
        }
        this->count = count;
    }
    void filter_block_uint16(uint16_pair **input)
    {
        for (int i = 0; i < numStreams; ++i)
            check(msosm_dedisp_filter_block_uint16(h_[i].h, input[i]), "filter_block_uint16");
    }
    void get_output(Complex **output)
    {
        for (int i = 0; i < numStreams; ++i) {
            out_.resize(h_[i].block() + 1);
            check(msosm_dedisp_get_output_c64(h_[i].h, out_.data()), "get_output");
            std::copy(out_.begin(), out_.end() - 1, output[i]);
        }
    }
    void synchronize()
    {
        for (auto &h : h_)
            check(msosm_dedisp_synchronize(h.h), "synchronize");
    }

    int count = 0;
    int numStreams;
    std::vector<unsigned long> M, M_min, Nd;
    std::vector<int> delaycount;
    std::vector<Complex *> output_buffer_d;

private:
    std::vector<float> bw_, dm_, f0_;
    std::vector<detail::Handle> h_;
    std::vector<Complex> out_;
};

// ---------------------------------------------------------------------------
// detection + folding (folding/include/fold_gpu.h:10-42)
// ---------------------------------------------------------------------------

class Fold_GPU {
public:
    Fold_GPU(float period, float fs, unsigned long size, std::string outfileName = "fold.txt",
             unsigned long time_bin = (unsigned long)-1)
        : size_(size), outfile_(std::move(outfileName))
    {
        check(msosm_fold_create(period, fs, size, time_bin, &h_), "msosm_fold_create");
        check(msosm_fold_get_shape(h_, &period_samples, &this->time_bin), "msosm_fold_get_shape");
        folded_.assign(this->time_bin, 0.f);
        folded_data = folded_.data();
        intensity_.assign(size, 0.f);
        total_intensity = intensity_.data();
    }
    Fold_GPU(const Fold_GPU &) = delete;
    Fold_GPU &operator=(const Fold_GPU &) = delete;
    ~Fold_GPU()
    {
        if (h_)
            msosm_fold_destroy(h_);
    }
    void discard_samples(unsigned long Nd) { check(msosm_fold_discard_samples(h_, Nd), "discard_samples"); }
    // MSOSM_GPU_BATCH / OSM_GPU_BATCH: ordered after their last filter call
    void calculate_intensity(MSOSM_GPU_BATCH *pol1, MSOSM_GPU_BATCH *pol2)
    {
        check(msosm_fold_calculate_intensity_dedisp(h_, pol1->handle(), pol2 ? pol2->handle() : nullptr),
              "calculate_intensity");
    }
    // any other class with a device output_buffer_d (waits for the device)
    template <typename T>
    void calculate_intensity(T *pol1, T *pol2)
    {
        check(msosm_fold_calculate_intensity(h_, pol1->output_buffer_d, pol2 ? pol2->output_buffer_d : nullptr),
              "calculate_intensity");
    }
    // the host total_intensity buffer, after the caller filled it
    void load_total_intensity() { check(msosm_fold_set_intensity(h_, total_intensity), "set_intensity"); }
    void fold_data() { check(msosm_fold_data(h_), "fold_data"); }
    void fold_data_bins() { check(msosm_fold_data_bins(h_, folded_data), "fold_data_bins"); }
    void write_to_file()
    {
        FILE *f = std::fopen(outfile_.c_str(), "w");
        if (!f)
            return;
        for (unsigned long i = 0; i < time_bin; ++i)
            std::fprintf(f, "%g\n", folded_data[i]);
        std::fclose(f);
    }

    float *folded_data = nullptr;
    unsigned long time_bin = 0;
    float *total_intensity = nullptr;
    unsigned long period_samples = 0;

private:
    msosm_fold *h_ = nullptr;
    unsigned long size_;
    std::string outfile_;
    std::vector<float> folded_, intensity_;
};

// ---------------------------------------------------------------------------
// psrdada/include/psrdada.h:17-43 -- a PSRDADA file (msosm_dada_*)
// ---------------------------------------------------------------------------

class PSRDADA {
public:
    explicit PSRDADA(std::string filename) : infileName(std::move(filename))
    {
        check(msosm_dada_open(infileName.c_str(), &h_), "PSRDADA");
        msosm_dada_info info;
        check(msosm_dada_get_info(h_, &info), "PSRDADA");
        check(msosm_dada_get_header(h_, headerBuffer), "PSRDADA");
        filesize = (unsigned long)info.filesize;
        bw = info.bw;
        fc = info.fc;
        nbit = info.nbit;
        nchan = info.nchan;
        ndim = info.ndim;
        npol = info.npol;
        outfileName = infileName.substr(0, infileName.find_last_of('.')) + "_dedisp_folded.txt";
        std::printf("%g %g %d %d %d %d\n", bw, fc, nbit, nchan, ndim, npol);
    }
    PSRDADA(const PSRDADA &) = delete;
    PSRDADA &operator=(const PSRDADA &) = delete;
    ~PSRDADA()
    {
        if (h_)
            msosm_dada_close(h_);
    }
    // n: samples per polarisation and read, a multiple of 2048
    void initBuffer(size_t n)
    {
        if (n % 2048 != 0)
            check(MSOSM_ERR_BAD_ARG, "initBuffer: n must be a multiple of frameSamples (2048)");
        pol1_.assign(n, uint16_pair{0, 0});
        pol2_.assign(n, uint16_pair{0, 0});
        pol1_in = pol1_.data();
        pol2_in = pol2_.data();
        frameCount = (int)(n / 2048);
        check(msosm_dada_read_count(h_, n, &readCount), "initBuffer");
    }
    void readSamples() { check(msosm_dada_read(h_, pol1_.size(), pol1_in, pol2_in), "readSamples"); }

    char headerBuffer[4096] = {0};
    std::string infileName;
    unsigned long filesize = 0;
    unsigned long readCount = 0;
    std::string outfileName;
    float bw = 0.f;
    float fc = 0.f;
    int nbit = 0;
    int nchan = 0;
    int ndim = 0;
    int npol = 0;
    int hdr_size = 4096;
    uint16_pair *pol1_in = nullptr;
    uint16_pair *pol2_in = nullptr;
    int frameCount = 0;

private:
    msosm_dada *h_ = nullptr;
    std::vector<uint16_pair> pol1_, pol2_;
};

// ---------------------------------------------------------------------------
// Not a reference class: the output-file thread of the reference's drivers
// (multiple_dm_concurrent_msosm.cpp:80-146: each call's numDMs * count * M
// uint16 pairs appended to "<date time>_<numDMs>.bin") as an object over
// msosm_writer_*.  push() after each filter call replaces get_output_thread
// plus the wait_for_threads handshake; no busy-wait.
// ---------------------------------------------------------------------------

class SeriesFileWriter {
public:
    template <class Dedisperser>
    SeriesFileWriter(Dedisperser &d, const std::string &path, int kind = MSOSM_WRITE_UINT16, int depth = 2,
                     int threads = 1)
    {
        check(msosm_writer_create(d.handle(), path.c_str(), kind, depth, threads, &w_), "SeriesFileWriter");
    }
    SeriesFileWriter(const SeriesFileWriter &) = delete;
    SeriesFileWriter &operator=(const SeriesFileWriter &) = delete;
    ~SeriesFileWriter() { close(); }
    void push() { check(msosm_writer_push(w_), "SeriesFileWriter::push"); }
    unsigned long long close()
    {
        if (w_) {
            msosm_writer *w = w_;
            w_ = nullptr;
            check(msosm_writer_close(w, &bytes_), "SeriesFileWriter::close");
        }
        return bytes_;
    }
    // the reference writer's file name: local date and time, the trial count
    static std::string reference_name(int numDMs)
    {
        char buf[64];
        std::time_t t = std::time(nullptr);
        std::strftime(buf, sizeof buf, "%Y-%m-%d %H:%M:%S", std::localtime(&t));
        return std::string(buf) + "_" + std::to_string(numDMs) + ".bin";
    }

private:
    msosm_writer *w_ = nullptr;
    unsigned long long bytes_ = 0;
};

// ---------------------------------------------------------------------------
// simulated_pulsar/include/AWGN.h:8-31 -- complex white Gaussian noise
// (msosm_sim_awgn).  `seed` replaces the reference's default-seeded engine.
// ---------------------------------------------------------------------------

class AWGN {
public:
    AWGN() : mean(0.f), variance(1.f), numberOfSamples(100), isSNRMode(false) {}
    AWGN(float mean_, float variance_, unsigned long n)
        : mean(mean_), variance(variance_), numberOfSamples(n), isSNRMode(false)
    {
    }
    AWGN(float SNR, unsigned long n) : mean(0.f), variance(1.f), numberOfSamples(n), isSNRMode(true), snr(SNR) {}
    AWGN(const AWGN &) = delete;
    AWGN &operator=(const AWGN &) = delete;
    ~AWGN() { deallocate(); }

    // numberOfSamples complex values in host memory owned by this object
    // until deallocate()
    Complex *generateNoiseSamples()
    {
        deallocate();
        check(msosm_host_alloc(sizeof(Complex) * numberOfSamples, 0, (void **)&samples), "generateNoiseSamples");
        check(msosm_sim_awgn(seed, numberOfSamples, isSNRMode ? 1 : 0, mean, variance, snr, samples),
              "generateNoiseSamples");
        return samples;
    }
    void deallocate()
    {
        if (samples)
            msosm_host_free(samples, 0);
        samples = nullptr;
    }

    unsigned long long seed = 0;

private:
    float mean, variance;
    unsigned long numberOfSamples;
    bool isSNRMode;
    float snr = 0.f;
    Complex *samples = nullptr;
};

// ---------------------------------------------------------------------------
// simulated_pulsar/include/simulated_complex_signal.h:9-63 -- two deltas per
// period dispersed at DM, tiled, optional AWGN and uint16 codec, generated on
// the GPU (msosm_sim_two_spike).  The plot_abs methods (matplotlib) are not
// provided.
// ---------------------------------------------------------------------------

class SimulatedComplexSignal {
public:
    SimulatedComplexSignal(float bw_, float dm_, float f0_, float period_, std::string mode = "complex")
        : data_type(std::move(mode)), bw(bw_), fs(bw_), kdm(4.15e15f), dm(dm_), f0(f0_), period(period_)
    {
        msosm_sim_two_spike_info info;
        check(msosm_sim_two_spike_shape(bw, dm, f0, period, &info), "SimulatedComplexSignal");
        Np = info.Np;
        Nd = info.Nd;
        range = info.range;
        check(msosm_prepare_min_order_msosm(Nd, &M_min), "SimulatedComplexSignal");
        M = M_min;
    }
    SimulatedComplexSignal(const SimulatedComplexSignal &) = delete;
    SimulatedComplexSignal &operator=(const SimulatedComplexSignal &) = delete;
    ~SimulatedComplexSignal() { release(); }

    void generate_pulsar_signal(unsigned long repeat = 1, bool add_noise = false, float SNR = 0, bool pinned = true)
    {
        release();
        pinned_ = pinned;
        signal_size = repeat * Np;
        check(msosm_host_alloc(sizeof(Complex) * signal_size, pinned ? 1 : 0, (void **)&signal),
              "generate_pulsar_signal");
        if (data_type == "uint16")
            check(msosm_host_alloc(sizeof(uint16_pair) * signal_size, pinned ? 1 : 0, (void **)&signal_u16),
                  "generate_pulsar_signal");
        check(msosm_sim_two_spike(bw, dm, f0, period, repeat, add_noise ? 1 : 0, SNR, seed, signal, signal_u16,
                                  &signal_power),
              "generate_pulsar_signal");
    }

    Complex *signal = nullptr;
    uint16_pair *signal_u16 = nullptr;
    std::string data_type;
    unsigned long signal_size = 0;
    unsigned long Np = 0;
    unsigned long Nd = 0;
    unsigned long M = 0;
    unsigned long M_min = 0;
    unsigned long range = 0;
    // not in the reference's public fields
    float signal_power = 0.f;  // dB, measured over one period
    unsigned long long seed = 0;

private:
    void release()
    {
        if (signal)
            msosm_host_free(signal, pinned_ ? 1 : 0);
        if (signal_u16)
            msosm_host_free(signal_u16, pinned_ ? 1 : 0);
        signal = nullptr;
        signal_u16 = nullptr;
    }
    float bw, fs, kdm, dm, f0, period;
    bool pinned_ = true;
};

}  // namespace msosm_b200
