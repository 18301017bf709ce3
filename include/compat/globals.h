// globals.h -- include-name compatibility header: a program written against
// the reference (utils/include/globals.h) compiles unchanged with
// `-I include/compat -I include` and links -lmsosm_b200 -lcudart.
//
// What the reference's globals.h gave its drivers: the standard headers they
// rely on, `using namespace std`, uint16_pair and Complex, the `verbose`
// flag, pi, and the plotting helpers (matplotlib-cpp).  There is no display
// here: the plot helpers are headless.  With MSOSM_PLOT_DUMP set to a path,
// every plotted series is appended to that file as a record (the helper's
// name, the element count, then the values as float32: |x| for plot_abs, the
// two components for plot_pol1/plot_pol2 of uint16 pairs, decoded
// offset-binary); otherwise they do nothing.  show() does nothing.
#pragma once

#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <getopt.h>
#include <iomanip>
#include <iostream>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <unistd.h>
#include <vector>

#include <cuda_runtime_api.h>
#include <nvtx3/nvToolsExt.h>

#include "matplotlibcpp.h"
#include "msosm_gpu_b200.hpp"

using namespace std;
namespace plt = matplotlibcpp;

using msosm_b200::Complex;
using msosm_b200::uint16_pair;

inline bool verbose = false;
constexpr auto pi = M_PI;

namespace msosm_b200 {
namespace compat {

// one record: 32-byte name, uint64 count, count float32 values
inline void dump(const char *name, const std::vector<float> &v)
{
    const char *path = std::getenv("MSOSM_PLOT_DUMP");
    if (!path || !*path)
        return;
    FILE *f = std::fopen(path, "ab");
    if (!f)
        return;
    char n[32] = {0};
    std::strncpy(n, name, 31);
    const uint64_t c = v.size();
    std::fwrite(n, 1, 32, f);
    std::fwrite(&c, 8, 1, f);
    if (c)
        std::fwrite(v.data(), sizeof(float), c, f);
    std::fclose(f);
}

// offset-binary sample as the reference's uint16ToComplex decodes it
inline float decode(uint16_t v) { return v == 0 ? 0.f : (float)((int)v - 32768); }

}  // namespace compat
}  // namespace msosm_b200

inline void banner() { std::cout << "==================================================" << std::endl; }
inline void line() { std::cout << "--------------------------------------------------" << std::endl; }
inline void show() {}

inline void plot_abs(uint16_pair *signal, unsigned long size)
{
    std::vector<float> v(size);
    for (unsigned long i = 0; i < size; ++i)
        v[i] = std::hypot(msosm_b200::compat::decode(signal[i].first), msosm_b200::compat::decode(signal[i].second));
    msosm_b200::compat::dump("plot_abs_u16", v);
}
inline void plot_abs(Complex *signal, unsigned long size)
{
    std::vector<float> v(size);
    for (unsigned long i = 0; i < size; ++i)
        v[i] = std::hypot(signal[i].x, signal[i].y);
    msosm_b200::compat::dump("plot_abs_c64", v);
}
inline void plot_pol1(uint16_pair *signal, unsigned long size)
{
    std::vector<float> v(size);
    for (unsigned long i = 0; i < size; ++i)
        v[i] = msosm_b200::compat::decode(signal[i].first);
    msosm_b200::compat::dump("plot_pol1", v);
}
inline void plot_pol2(uint16_pair *signal, unsigned long size)
{
    std::vector<float> v(size);
    for (unsigned long i = 0; i < size; ++i)
        v[i] = msosm_b200::compat::decode(signal[i].second);
    msosm_b200::compat::dump("plot_pol2", v);
}
template <typename T>
inline void plot(T *signal, unsigned long size)
{
    std::vector<float> v(size);
    for (unsigned long i = 0; i < size; ++i)
        v[i] = (float)signal[i];
    msosm_b200::compat::dump("plot", v);
}
// the reference plots |x| of trial `index` (or of every trial) of one block
inline void plot_abs_concurrent(Complex *signal, unsigned long block_size, unsigned long size, int numDMs, int index)
{
    (void)numDMs;
    std::vector<float> v(size);
    for (unsigned long i = 0; i < size; ++i)
        v[i] = std::hypot(signal[(size_t)index * block_size + i].x, signal[(size_t)index * block_size + i].y);
    msosm_b200::compat::dump("plot_abs_concurrent", v);
}
inline void plot_abs_concurrent_all(Complex *signal, int block_size, unsigned long size, int numDMs)
{
    for (int i = 0; i < numDMs; ++i)
        plot_abs_concurrent(signal, (unsigned long)block_size, size, numDMs, i);
}
