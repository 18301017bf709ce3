// dada.cpp -- PSRDADA baseband files (the C ABI's msosm_dada_*).
//
// Format, as the reference reads it (psrdada/psrdada.cpp:3-94,
// psrdada/include/psrdada.h:11-12): a 4096-byte ASCII header of "KEY value"
// lines (NUL padded), then frames of 2048 uint16 pairs of polarisation 1
// followed by 2048 pairs of polarisation 2.  The header keys the pipeline
// uses are BW (MHz), FREQ (centre, MHz), NBIT, NCHAN, NDIM, NPOL; a line is
// split at its first space and the value starts at the next non-space
// character, as the reference splits it (psrdada.cpp:96-113).
#include "msosm_b200.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>

#include "kernels.hpp"

namespace {

constexpr size_t kHeaderBytes = 4096;
constexpr unsigned long kFrameSamples = 2048;

msosm_status dada_fail(msosm_status s, const std::string &msg)
{
    msosm::set_error_message(msg.c_str());
    return s;
}

}  // namespace

struct msosm_dada {
    std::FILE *f = nullptr;
    char header[kHeaderBytes + 1] = {0};
    msosm_dada_info info{};
};

namespace {

void parse_header(msosm_dada *d)
{
    // the header text ends at its first NUL
    const std::string text(d->header, strnlen(d->header, kHeaderBytes));
    size_t pos = 0;
    while (pos < text.size()) {
        size_t eol = text.find('\n', pos);
        if (eol == std::string::npos)
            eol = text.size();
        const std::string line = text.substr(pos, eol - pos);
        pos = eol + 1;
        const size_t sp = line.find(' ');
        if (sp == std::string::npos)
            continue;
        const std::string key = line.substr(0, sp);
        const size_t vs = line.find_first_not_of(' ', sp);
        if (vs == std::string::npos)
            continue;
        const char *v = line.c_str() + vs;
        if (key == "BW") {
            d->info.bw = std::strtof(v, nullptr);
            d->info.have |= MSOSM_DADA_HAVE_BW;
        } else if (key == "FREQ") {
            d->info.fc = std::strtof(v, nullptr);
            d->info.have |= MSOSM_DADA_HAVE_FREQ;
        } else if (key == "NBIT") {
            d->info.nbit = (int)std::strtol(v, nullptr, 10);
        } else if (key == "NCHAN") {
            d->info.nchan = (int)std::strtol(v, nullptr, 10);
        } else if (key == "NDIM") {
            d->info.ndim = (int)std::strtol(v, nullptr, 10);
        } else if (key == "NPOL") {
            d->info.npol = (int)std::strtol(v, nullptr, 10);
        }
    }
}

}  // namespace

extern "C" {

msosm_status msosm_dada_open(const char *path, msosm_dada **out)
{
    if (!path || !out)
        return dada_fail(MSOSM_ERR_BAD_ARG, "msosm_dada_open: null argument");
    *out = nullptr;
    std::FILE *f = std::fopen(path, "rb");
    if (!f)
        return dada_fail(MSOSM_ERR_BAD_ARG, std::string("cannot open file: ") + path);
    msosm_dada *d = new (std::nothrow) msosm_dada;
    if (!d) {
        std::fclose(f);
        return dada_fail(MSOSM_ERR_OOM, "host allocation");
    }
    d->f = f;
    if (std::fseek(f, 0, SEEK_END) != 0) {
        msosm_dada_close(d);
        return dada_fail(MSOSM_ERR_BAD_ARG, "cannot seek the file");
    }
    const long size = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (size < (long)kHeaderBytes || std::fread(d->header, 1, kHeaderBytes, f) != kHeaderBytes) {
        msosm_dada_close(d);
        return dada_fail(MSOSM_ERR_BAD_ARG, "file shorter than its 4096-byte header");
    }
    d->info.filesize = (unsigned long long)size;
    parse_header(d);
    *out = d;
    return MSOSM_OK;
}

msosm_status msosm_dada_close(msosm_dada *d)
{
    if (d) {
        if (d->f)
            std::fclose(d->f);
        delete d;
    }
    return MSOSM_OK;
}

msosm_status msosm_dada_get_info(const msosm_dada *d, msosm_dada_info *info)
{
    if (!d || !info)
        return dada_fail(MSOSM_ERR_BAD_ARG, "null argument");
    *info = d->info;
    return MSOSM_OK;
}

msosm_status msosm_dada_get_header(const msosm_dada *d, char *header)
{
    if (!d || !header)
        return dada_fail(MSOSM_ERR_BAD_ARG, "null argument");
    std::memcpy(header, d->header, kHeaderBytes);
    return MSOSM_OK;
}

msosm_status msosm_dada_read_count(const msosm_dada *d, unsigned long n, unsigned long *count)
{
    if (!d || !count || n == 0 || n % kFrameSamples != 0)
        return dada_fail(MSOSM_ERR_BAD_ARG, "n must be a positive multiple of 2048 samples");
    *count = (unsigned long)((d->info.filesize - kHeaderBytes) / (2ull * n * sizeof(msosm_uint16_pair)));
    return MSOSM_OK;
}

msosm_status msosm_dada_read(msosm_dada *d, unsigned long n, msosm_uint16_pair *pol1, msosm_uint16_pair *pol2)
{
    if (!d || !pol1 || !pol2 || n == 0 || n % kFrameSamples != 0)
        return dada_fail(MSOSM_ERR_BAD_ARG, "n must be a positive multiple of 2048 samples; buffers non-null");
    const long at = std::ftell(d->f);
    if (at < 0 || (unsigned long long)at + 2ull * n * sizeof(msosm_uint16_pair) > d->info.filesize)
        return dada_fail(MSOSM_ERR_STATE, "end of file: fewer than 2 x n samples left");
    for (unsigned long fr = 0; fr < n / kFrameSamples; ++fr) {
        if (std::fread(pol1 + fr * kFrameSamples, sizeof(msosm_uint16_pair), kFrameSamples, d->f) != kFrameSamples ||
            std::fread(pol2 + fr * kFrameSamples, sizeof(msosm_uint16_pair), kFrameSamples, d->f) != kFrameSamples)
            return dada_fail(MSOSM_ERR_STATE, "short read");
    }
    return MSOSM_OK;
}

}  // extern "C"
