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
//  * get_output() waits for the copy, so the wait_for_cpu flag of the
//    reference (a busy-wait on a plain bool, msosm_gpu_dm_concurrent.cpp:
//    156-160) is kept as a field but never spun on; get_output_thread keeps
//    the hand-over to an output thread through wait_for_threads (atomic
//    flags, a yielding wait bounded at 60 s);
//  * copies of an object share its device handle (the reference's shallow
//    copies share its device buffers);
//  * trials with DM 0 get all block delays 0 (undefined in the reference).
#pragma once

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <ctime>
#include <cstdlib>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "msosm_b200.h"

namespace msosm_b200 {

using Complex = msosm_complex;
using uint16_pair = msosm_uint16_pair;

// Not in the reference: MS-OSM objects initialised after use_tensor_cores(true)
// run their inverse transforms on the tensor cores (MSOSM_FLAG_TENSOR_F16: f16
// operands, f32 accumulation, FFT sizes 4096, 8192 and 16384; series error ~5e-4
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

// One msosm_dedisp handle plus the reference-shaped views of its state,
// shared by every copy of the object that holds it: the reference's classes
// copy shallowly (their device buffers are shared by the copies, e.g. an
// object passed by value to a thread, multiple_thread_osm.cpp:5-13), and so
// do these.  The handle is destroyed with the last copy, or by reset().
struct HandleState {
    HandleState() = default;
    HandleState(const HandleState &) = delete;
    HandleState &operator=(const HandleState &) = delete;
    ~HandleState()
    {
        if (h)
            msosm_dedisp_destroy(h);
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

class Handle {
public:
    void create(const float *bw, const float *dm, const float *f0, int n, unsigned long fftpoint, int count,
                unsigned long input_size, unsigned int flags)
    {
        auto st = std::make_shared<HandleState>();
        check(msosm_dedisp_create(bw, dm, f0, n, fftpoint, count, input_size, flags, &st->h),
              "msosm_dedisp_create");
        check(msosm_dedisp_get_info(st->h, &st->info), "msosm_dedisp_get_info");
        st->n_ = n;
        st->Nd.resize(n);
        st->delaycount.resize(n);
        check(msosm_dedisp_get_nd(st->h, st->Nd.data()), "msosm_dedisp_get_nd");
        check(msosm_dedisp_get_delaycount(st->h, st->delaycount.data()), "msosm_dedisp_get_delaycount");
        const unsigned long fp = st->info.fftpoint;
        st->dp.assign((size_t)n * fp, 0);
        st->H.assign((size_t)n * fp, Complex{0.f, 0.f});
        for (int i = 0; i < n; ++i) {
            check(msosm_dedisp_get_delay_points(st->h, i, st->dp.data() + (size_t)i * fp), "delay_points");
            check(msosm_dedisp_get_dedisp_params(st->h, i, st->H.data() + (size_t)i * fp), "dedisp_params");
        }
        s_ = std::move(st);
    }
    // releases the device handle for every copy (the reference's reset_device
    // resets the whole device)
    void reset()
    {
        if (s_ && s_->h) {
            msosm_dedisp_destroy(s_->h);
            s_->h = nullptr;
        }
    }
    HandleState *operator->() const
    {
        if (!s_)
            check(MSOSM_ERR_STATE, "object used before initialize_uint16");
        return s_.get();
    }

private:
    std::shared_ptr<HandleState> s_;
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
        M = h_->info.M;
        M_min = h_->info.M_min;
        this->count = h_->info.count;
        delaycount = h_->delaycount[0];
        delay_points = h_->dp.data();
        dedisp_params = h_->H.data();
        output_buffer_d = h_->device_output();
    }
    void filter_block_uint16(uint16_pair *input)
    {
        check(msosm_dedisp_filter_block_uint16(h_->h, input), "filter_block_uint16");
    }
    void get_output(Complex *output)
    {
        // the handle's buffer ends with one extra element; copy count*M
        out_.resize(h_->block() + 1);
        check(msosm_dedisp_get_output_c64(h_->h, out_.data()), "get_output");
        std::copy(out_.begin(), out_.end() - 1, output);
    }

    int count = 0;
    Complex *output_buffer_d = nullptr;
    msosm_dedisp *handle() const { return h_->h; }

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
        M = h_->info.M;
        M_min = h_->info.M_min;
        this->count = h_->info.count;
        dedisp_params = h_->H.data();
        output_buffer_d = h_->device_output();
        total_memory = h_->info.device_bytes;
    }
    unsigned long total_memory = 0;
};

// ---------------------------------------------------------------------------
// many DMs over one input (dedispersion/include/msosm_gpu_concurrent.h:15-64)
// ---------------------------------------------------------------------------

class MSOSM_GPU_DM_concurrent {
public:
    // Prepare_MSOSM_DM_concurrent's constructor (msosm_prepare_dm_concurrent.cpp:3-29):
    // the smear Nd of every trial; M, M_min, delaycount, dedisp_params and
    // delay_points are allocated here and filled by the methods below or by
    // initialize_uint16
    MSOSM_GPU_DM_concurrent(float *bw, float *dm, float *f0, int numDMs)
        : numDMs(numDMs), bw_(bw, bw + numDMs), dm_(dm, dm + numDMs), f0_(f0, f0 + numDMs), nd_(numDMs, 0),
          m_(numDMs, 0), m_min_(numDMs, 0), dc_(numDMs, 0), dp_ptr_(numDMs, nullptr), h_ptr_(numDMs, nullptr),
          dp_own_(numDMs), h_own_(numDMs)
    {
        for (int i = 0; i < numDMs; ++i)
            check(msosm_prepare_nd(bw[i], dm[i], f0[i], &nd_[i]), "msosm_prepare_nd");
        bind();
    }
    MSOSM_GPU_DM_concurrent(const MSOSM_GPU_DM_concurrent &) = delete;
    MSOSM_GPU_DM_concurrent &operator=(const MSOSM_GPU_DM_concurrent &) = delete;
    virtual ~MSOSM_GPU_DM_concurrent() = default;
    void get_device_info() { std::printf("CUDA devices: %d\n", msosm_device_count()); }

    // --- Prepare_MSOSM_DM_concurrent (dedispersion/include/prepare_concurrent.h:10-38)
    // per-trial minimum orders; M_common = M_common_min = their largest
    // (msosm_prepare_dm_concurrent.cpp:31-49)
    void calculate_min_order()
    {
        M_common = 0;
        for (int i = 0; i < numDMs; ++i) {
            check(osm_ ? msosm_prepare_min_order_osm(nd_[i], &m_[i]) : msosm_prepare_min_order_msosm(nd_[i], &m_[i]),
                  "calculate_min_order");
            m_min_[i] = m_[i];
            M_common = std::max(M_common, m_[i]);
        }
        M_common_min = M_common;
    }
    void override_order(unsigned long order) { M_common = order; }
    // trial i's filter at the common order (msosm_prepare_dm_concurrent.cpp:56-103)
    void generate_dedisp_params(int i)
    {
        h_own_[i].assign(2 * M_common, Complex{0.f, 0.f});
        check(msosm_prepare_dedisp_params(bw_[i], dm_[i], f0_[i], M_common, h_own_[i].data()),
              "generate_dedisp_params");
        h_ptr_[i] = h_own_[i].data();
    }
    // trial i's block delays at the common order (msosm_prepare_dm_concurrent.cpp:105-168)
    void segmentation(int i)
    {
        dp_own_[i].assign(2 * M_common, 0);
        check(msosm_prepare_segmentation(bw_[i], dm_[i], f0_[i], M_common, &dc_[i], dp_own_[i].data()),
              "segmentation");
        dp_ptr_[i] = dp_own_[i].data();
    }

    // --- MSOSM_GPU_DM_concurrent (dedispersion/include/msosm_gpu_concurrent.h:15-64)
    void initialize_uint16(unsigned long fftpoint, int count = 1, unsigned long input_size = 0,
                           bool compute_only = false)
    {
        create(fftpoint, count, input_size, extra_flags());
        this->compute_only = compute_only;
    }
    void initialize_threads_flag(int thread_num)
    {
        threads_flag_.reset(new std::atomic<bool>[thread_num > 0 ? thread_num : 1]());
        wait_for_threads = threads_flag_.get();
    }
    void filter_block_uint16(uint16_pair *input)
    {
        check(msosm_dedisp_filter_block_uint16(h_->h, input), "filter_block_uint16");
    }
    // numDMs*count*M + 1 elements, [dm][count*M] then a trailing zero
    void get_output(Complex *output) { check(msosm_dedisp_get_output_c64(h_->h, output), "get_output"); }
    void get_output(uint16_pair *output)
    {
        check(msosm_dedisp_get_output_uint16(h_->h, output), "get_output");
    }
    // The reference's hand-over to an output thread
    // (msosm_gpu_dm_concurrent.cpp:182-195): unless compute_only, wait until
    // that thread has taken the previous batch (it clears
    // wait_for_threads[thread_id]), mark the slot taken, copy.  The wait
    // yields instead of spinning on a plain bool and gives up after 60 s.
    void get_output_thread(uint16_pair *output, int thread_id)
    {
        if (!compute_only && wait_for_threads) {
            const auto t0 = std::chrono::steady_clock::now();
            while (wait_for_threads[thread_id].load(std::memory_order_acquire)) {
                if (std::chrono::steady_clock::now() - t0 > std::chrono::seconds(60))
                    check(MSOSM_ERR_TIMEOUT, "get_output_thread: the output thread did not take the last batch");
                std::this_thread::yield();
            }
            wait_for_threads[thread_id].store(true, std::memory_order_release);
        }
        get_output(output);
    }
    void synchronize() { check(msosm_dedisp_synchronize(h_->h), "synchronize"); }
    void reset_device() { h_.reset(); }
    msosm_dedisp *handle() const { return h_->h; }

    int count = 0;
    bool wait_for_cpu = false;
    std::atomic<bool> *wait_for_threads = nullptr;  // one flag per output thread
    unsigned long M_common = 0, M_common_min = 0;
    // per trial (arrays of numDMs), as Prepare_MSOSM_DM_concurrent holds them
    unsigned long *M = nullptr, *M_min = nullptr;
    int *delaycount = nullptr;
    Complex **dedisp_params = nullptr;  // [numDMs] -> 2*M_common filter values
    int **delay_points = nullptr;       // [numDMs] -> 2*M_common block delays
    unsigned long *Nd = nullptr;
    int numDMs;
    // the same per-trial views by index
    int *delay_points_of(int i) { return delay_points[i]; }
    Complex *dedisp_params_of(int i) { return dedisp_params[i]; }

protected:
    void create(unsigned long fftpoint, int count, unsigned long input_size, unsigned int flags)
    {
        h_.create(bw_.data(), dm_.data(), f0_.data(), numDMs, fftpoint, count, input_size, flags);
        calculate_min_order();
        this->count = h_->info.count;
        M_common = h_->info.M;
        M_common_min = h_->info.M_min;
        for (int i = 0; i < numDMs; ++i) {
            nd_[i] = h_->Nd[i];
            dc_[i] = h_->delaycount[i];
            dp_ptr_[i] = h_->dp.data() + (size_t)i * h_->info.fftpoint;
            h_ptr_[i] = h_->H.data() + (size_t)i * h_->info.fftpoint;
        }
    }
    void bind()
    {
        Nd = nd_.data();
        M = m_.data();
        M_min = m_min_.data();
        delaycount = dc_.data();
        delay_points = dp_ptr_.data();
        dedisp_params = h_ptr_.data();
    }
    bool compute_only = false;
    bool osm_ = false;  // Prepare_OSM_DM_concurrent's orders (osm_prepare_dm_concurrent.cpp)
    std::vector<float> bw_, dm_, f0_;
    std::vector<unsigned long> nd_, m_, m_min_;
    std::vector<int> dc_;
    std::vector<int *> dp_ptr_;
    std::vector<Complex *> h_ptr_;
    std::vector<std::vector<int>> dp_own_;
    std::vector<std::vector<Complex>> h_own_;
    std::unique_ptr<std::atomic<bool>[]> threads_flag_;
    detail::Handle h_;
};

// dedispersion/include/osm_gpu_concurrent.h:7-42
class OSM_GPU_DM_concurrent : public MSOSM_GPU_DM_concurrent {
public:
    using MSOSM_GPU_DM_concurrent::MSOSM_GPU_DM_concurrent;
    void initialize_uint16(unsigned long fftpoint = 0, int count = 1, bool compute_only = false)
    {
        osm_ = true;
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
        this->count = h_->info.count;
        M_loop = h_->info.M;
        M_loop_min = h_->info.M_min;
        Nd = h_->Nd;
        delaycount = h_->delaycount;
    }
    // every trial is dedispersed here; filter_block_uint16(out, i) then
    // copies trial i (the reference runs trial i's filter at that point)
    void input_process(uint16_pair *input)
    {
        check(msosm_dedisp_filter_block_uint16(h_->h, input), "input_process");
        all_.resize((size_t)numOutput * h_->block() + 1);
        check(msosm_dedisp_get_output_c64(h_->h, all_.data()), "get_output");
    }
    void filter_block_uint16(Complex **output, int i)
    {
        std::copy(all_.begin() + (size_t)i * h_->block(), all_.begin() + (size_t)(i + 1) * h_->block(), output[i]);
    }
    void synchronize() { check(msosm_dedisp_synchronize(h_->h), "synchronize"); }

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
        flags_.reset(new bool[numStreams > 0 ? numStreams : 1]());
        wait_for_cpu = flags_.get();
    }
    void get_output(Complex **output)
    {
        all_.resize((size_t)numStreams * block() + 1);
        check(msosm_dedisp_get_output_c64(h_->h, all_.data()), "get_output");
        for (int i = 0; i < numStreams; ++i)
            std::copy(all_.begin() + (size_t)i * block(), all_.begin() + (size_t)(i + 1) * block(), output[i]);
    }
    void get_output(uint16_pair **output)
    {
        u_.resize((size_t)numStreams * block() + 1);
        check(msosm_dedisp_get_output_uint16(h_->h, u_.data()), "get_output");
        for (int i = 0; i < numStreams; ++i)
            std::copy(u_.begin() + (size_t)i * block(), u_.begin() + (size_t)(i + 1) * block(), output[i]);
    }
    int numStreams;
    unsigned long M_stream = 0, M_stream_min = 0;
    // one flag per stream, as the reference's (msosm_gpu_batch_stream.h:73);
    // get_output waits for its copy, so nothing spins on them
    bool *wait_for_cpu = nullptr;

private:
    std::unique_ptr<bool[]> flags_;
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
            M[i] = h_[i]->info.M;
            M_min[i] = h_[i]->info.M_min;
            fftpoint[i] = h_[i]->info.fftpoint;
            Nd[i] = h_[i]->Nd[0];
            delaycount[i] = h_[i]->delaycount[0];
            output_buffer_d[i] = h_[i]->device_output();
        }
        this->count = count;
    }
    void filter_block_uint16(uint16_pair **input)
    {
        for (int i = 0; i < numStreams; ++i)
            check(msosm_dedisp_filter_block_uint16(h_[i]->h, input[i]), "filter_block_uint16");
    }
    void get_output(Complex **output)
    {
        for (int i = 0; i < numStreams; ++i) {
            out_.resize(h_[i]->block() + 1);
            check(msosm_dedisp_get_output_c64(h_[i]->h, out_.data()), "get_output");
            std::copy(out_.begin(), out_.end() - 1, output[i]);
        }
    }
    void synchronize()
    {
        for (auto &h : h_)
            check(msosm_dedisp_synchronize(h->h), "synchronize");
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
        count_.assign(period_samples, 0ul);
        tmp_.assign(period_samples, 0.f);
        fold_count = count_.data();
        tmp_fold = tmp_.data();
        period_ = period;
        fs_ = fs;
    }
    Fold_GPU(const Fold_GPU &) = delete;
    Fold_GPU &operator=(const Fold_GPU &) = delete;
    ~Fold_GPU()
    {
        if (h_)
            msosm_fold_destroy(h_);
        if (planner_)
            msosm_fold_planner_destroy(planner_);
    }
    void discard_samples(unsigned long Nd)
    {
        check(msosm_fold_discard_samples(h_, Nd), "discard_samples");
        discard_ = Nd;
    }
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
    void fold_data()
    {
        check(msosm_fold_data(h_), "fold_data");
        if (track_raw_state)
            track_chunk();
    }
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
    // Fold_GPU's raw-resolution state (fold_gpu.h:27-28), period_samples
    // each: fold_count[p] counts the nonzero intensities folded at phase p
    // (over every completed period; the reference counts only periods that
    // lie inside one chunk, fold_gpu.cpp:124-132), tmp_fold holds the
    // intensities of the period in progress.  The device fold needs neither,
    // so they are kept only with track_raw_state set before the first
    // fold_data (each chunk's intensities are then read back to the host).
    unsigned long *fold_count = nullptr;
    float *tmp_fold = nullptr;
    bool track_raw_state = false;

private:
    // the chunk's destinations from the same fold state machine the device
    // fold follows (msosm_fold_planner_chunk), applied to its intensities
    void track_chunk()
    {
        if (!planner_)
            check(msosm_fold_planner_create(period_, fs_, discard_, &planner_), "fold planner");
        dest_.resize(size_);
        unsigned long long done = 0;
        check(msosm_fold_planner_chunk(planner_, size_, dest_.data(), &done), "fold planner");
        check(msosm_fold_get_intensity(h_, total_intensity), "fold_data");
        if (tmp_nz_.size() != period_samples)
            tmp_nz_.assign(period_samples, 0);
        for (unsigned long i = 0; i < size_; ++i) {
            if (dest_[i] < 0)
                continue;
            const unsigned long ph = (unsigned long)(dest_[i] & 0xFFFFFFFFll);
            tmp_fold[ph] = total_intensity[i];
            tmp_nz_[ph] = total_intensity[i] != 0.f;
            if (ph + 1 == period_samples)  // the period is complete
                for (unsigned long p = 0; p < period_samples; ++p)
                    fold_count[p] += tmp_nz_[p];
        }
    }

    msosm_fold *h_ = nullptr;
    msosm_fold_planner *planner_ = nullptr;
    unsigned long size_;
    std::string outfile_;
    std::vector<float> folded_, intensity_;
    std::vector<unsigned long> count_;
    std::vector<float> tmp_;
    std::vector<unsigned char> tmp_nz_;
    std::vector<int64_t> dest_;
    float period_ = 0.f, fs_ = 0.f;
    unsigned long discard_ = 0;
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
