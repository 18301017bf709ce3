// writer.cpp -- dedispersed series to a file while the device keeps working
// (msosm_writer_* of msosm_b200.h).
//
// The reference drivers hand each call's uint16 output to a writer thread
// that appends it to a binary file (multiple_dm_concurrent_msosm.cpp:80-146),
// the two sides signalling through a busy-waited flag in the output buffer's
// trailing element.  Here a writer owns `depth` slots, each a device buffer
// and a pinned host buffer.  msosm_writer_push encodes the call's series into
// a free slot's device buffer on the handle's stream (so the next call's
// kernels may overwrite the series at once), copies it to the slot's host
// buffer on the writer's own copy stream (under the next call's compute) and
// queues the slot; one of `threads` writer threads waits on the copy's event,
// writes the slot at its batch's offset in the file (pwrite: the file's
// layout is the call order whatever thread writes a batch) and frees it.
// Waits are on events and condition variables; nothing spins.
#include "msosm_b200.h"

#include <condition_variable>
#include <cerrno>
#include <cstdio>
#include <deque>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>
#include <fcntl.h>
#include <unistd.h>

#include "kernels.hpp"

using namespace msosm;

namespace {

msosm_status wfail(msosm_status s, const std::string &msg)
{
    set_error_message(msg.c_str());
    return s;
}

msosm_status wcuda(cudaError_t e, const char *what)
{
    cudaGetLastError();
    return wfail(e == cudaErrorMemoryAllocation ? MSOSM_ERR_OOM : MSOSM_ERR_CUDA,
                 std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace

struct msosm_writer {
    struct Slot {
        void *dev = nullptr, *host = nullptr;
        cudaEvent_t encoded = nullptr, copied = nullptr;
        unsigned long long batch = 0;
    };
    msosm_dedisp *d = nullptr;
    int fd = -1;
    int kind = MSOSM_WRITE_UINT16;
    size_t n = 0, elem = 0;  // elements (numDMs * count * M) and bytes per element
    cudaStream_t copy = nullptr;
    std::vector<Slot> slots;
    std::deque<int> free_q, write_q;
    std::mutex mu;
    std::condition_variable cv;
    std::vector<std::thread> th;
    bool closing = false;
    msosm_status err = MSOSM_OK;
    std::string errmsg;
    unsigned long long bytes = 0, batches = 0, pushed = 0;

    // all of buf at byte offset off
    bool write_at(const void *buf, size_t len, unsigned long long off)
    {
        const char *p = static_cast<const char *>(buf);
        while (len > 0) {
            const ssize_t r = ::pwrite(fd, p, len, (off_t)off);
            if (r < 0 && errno == EINTR)
                continue;
            if (r <= 0)
                return false;
            p += r;
            len -= (size_t)r;
            off += (unsigned long long)r;
        }
        return true;
    }

    void run()
    {
        for (;;) {
            int s;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return !write_q.empty() || closing; });
                if (write_q.empty())
                    return;
                s = write_q.front();
                write_q.pop_front();
            }
            cudaError_t e = cudaEventSynchronize(slots[s].copied);
            bool ok = false;
            if (e == cudaSuccess)
                ok = write_at(slots[s].host, elem * n, slots[s].batch * (unsigned long long)(elem * n));
            std::lock_guard<std::mutex> lk(mu);
            if (e != cudaSuccess && err == MSOSM_OK) {
                err = MSOSM_ERR_CUDA;
                errmsg = std::string("writer copy: ") + cudaGetErrorString(e);
            } else if (e == cudaSuccess && !ok && err == MSOSM_OK) {
                err = MSOSM_ERR_STATE;
                errmsg = "writer: short write to the output file";
            } else if (e == cudaSuccess) {
                bytes += (unsigned long long)(elem * n);
                batches += 1;
            }
            free_q.push_back(s);
            cv.notify_all();
        }
    }

    void release()
    {
        for (Slot &s : slots) {
            if (s.dev)
                cudaFree(s.dev);
            if (s.host)
                cudaFreeHost(s.host);
            if (s.encoded)
                cudaEventDestroy(s.encoded);
            if (s.copied)
                cudaEventDestroy(s.copied);
        }
        slots.clear();
        if (copy)
            cudaStreamDestroy(copy);
        copy = nullptr;
        if (fd >= 0)
            ::close(fd);
        fd = -1;
    }
};

extern "C" {

msosm_status msosm_writer_create(msosm_dedisp *d, const char *path, int kind, int depth, int threads,
                                 msosm_writer **out)
{
    if (!d || !path || !out)
        return wfail(MSOSM_ERR_BAD_ARG, "msosm_writer_create: null argument");
    *out = nullptr;
    if (kind != MSOSM_WRITE_UINT16 && kind != MSOSM_WRITE_C64)
        return wfail(MSOSM_ERR_BAD_ARG, "msosm_writer_create: kind must be MSOSM_WRITE_UINT16 or _C64");
    if (depth < 1 || depth > 16)
        return wfail(MSOSM_ERR_BAD_ARG, "msosm_writer_create: depth must be 1 .. 16");
    if (threads < 1 || threads > depth)
        return wfail(MSOSM_ERR_BAD_ARG, "msosm_writer_create: threads must be 1 .. depth");
    msosm_dedisp_info info;
    msosm_status st = msosm_dedisp_get_info(d, &info);
    if (st != MSOSM_OK)
        return st;
    if (info.flags & MSOSM_FLAG_NO_SERIES)
        return wfail(MSOSM_ERR_STATE, "msosm_writer_create: handle created with MSOSM_FLAG_NO_SERIES");
    msosm_writer *w = new (std::nothrow) msosm_writer;
    if (!w)
        return wfail(MSOSM_ERR_OOM, "host allocation");
    w->d = d;
    w->kind = kind;
    w->n = (size_t)info.numDMs * (size_t)info.count * info.M;
    w->elem = kind == MSOSM_WRITE_UINT16 ? sizeof(msosm_uint16_pair) : sizeof(msosm_complex);
    w->fd = ::open(path, O_WRONLY | O_CREAT | O_TRUNC, 0644);
    if (w->fd < 0) {
        delete w;
        return wfail(MSOSM_ERR_BAD_ARG, std::string("cannot open for writing: ") + path);
    }
    cudaError_t e = cudaStreamCreateWithFlags(&w->copy, cudaStreamNonBlocking);
    w->slots.resize(depth);
    for (int i = 0; i < depth && e == cudaSuccess; ++i) {
        msosm_writer::Slot &s = w->slots[i];
        e = cudaMalloc(&s.dev, w->elem * w->n + 16);
        if (e == cudaSuccess)
            e = cudaMallocHost(&s.host, w->elem * w->n + 16);
        if (e == cudaSuccess)
            e = cudaEventCreateWithFlags(&s.encoded, cudaEventDisableTiming);
        if (e == cudaSuccess)
            e = cudaEventCreateWithFlags(&s.copied, cudaEventDisableTiming);
        w->free_q.push_back(i);
    }
    if (e != cudaSuccess) {
        w->release();
        delete w;
        return wcuda(e, "msosm_writer_create");
    }
    for (int t = 0; t < threads; ++t)
        w->th.emplace_back([w] { w->run(); });
    *out = w;
    return MSOSM_OK;
}

msosm_status msosm_writer_push(msosm_writer *w)
{
    if (!w)
        return wfail(MSOSM_ERR_BAD_ARG, "null writer");
    int s;
    {
        std::unique_lock<std::mutex> lk(w->mu);
        w->cv.wait(lk, [&] { return !w->free_q.empty() || w->err != MSOSM_OK; });
        if (w->err != MSOSM_OK)
            return wfail(w->err, w->errmsg);
        s = w->free_q.front();
        w->free_q.pop_front();
    }
    msosm_writer::Slot &sl = w->slots[s];
    sl.batch = w->pushed;
    msosm_complex *series = nullptr;
    msosm_status st = msosm_dedisp_output_device_ptr(w->d, &series);
    cudaStream_t hs = dedisp_stream(w->d);
    cudaError_t e = cudaSuccess;
    if (st == MSOSM_OK) {
        // on the handle's stream: after this call's kernels, before the next's
        if (w->kind == MSOSM_WRITE_UINT16)
            e = launch_encode_u16(reinterpret_cast<const float2 *>(series), static_cast<uint32_t *>(sl.dev), w->n,
                                  hs);
        else
            e = cudaMemcpyAsync(sl.dev, series, w->elem * w->n, cudaMemcpyDeviceToDevice, hs);
        if (e == cudaSuccess)
            e = cudaEventRecord(sl.encoded, hs);
        if (e == cudaSuccess)
            e = cudaStreamWaitEvent(w->copy, sl.encoded, 0);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(sl.host, sl.dev, w->elem * w->n, cudaMemcpyDeviceToHost, w->copy);
        if (e == cudaSuccess)
            e = cudaEventRecord(sl.copied, w->copy);
    }
    std::lock_guard<std::mutex> lk(w->mu);
    if (st != MSOSM_OK || e != cudaSuccess) {
        w->free_q.push_front(s);
        return st != MSOSM_OK ? st : wcuda(e, "msosm_writer_push");
    }
    w->write_q.push_back(s);
    w->pushed += 1;
    w->cv.notify_all();
    return MSOSM_OK;
}

msosm_status msosm_writer_close(msosm_writer *w, unsigned long long *bytes_written)
{
    if (!w)
        return MSOSM_OK;
    {
        std::lock_guard<std::mutex> lk(w->mu);
        w->closing = true;
        w->cv.notify_all();
    }
    for (std::thread &t : w->th)
        if (t.joinable())
            t.join();
    msosm_status st = w->err;
    std::string msg = w->errmsg;
    if (bytes_written)
        *bytes_written = w->bytes;
    w->release();
    delete w;
    return st == MSOSM_OK ? MSOSM_OK : wfail(st, msg);
}

}  // extern "C"
