// host_prepare.cpp -- see host_prepare.hpp.
#include "host_prepare.hpp"

#include <cmath>

namespace msosm {

unsigned long dispersion_smear(float bw, float dm, float f0)
{
    // Nd = floor(kdm*dm*(1/pow(f0,2) - 1/pow(f0+bw,2)) / (1/fs)), fs = bw:
    // kdm*dm and f0+bw are float operations, 1/fs a float quotient, the rest
    // double (msosm_prepare.cpp:5-8).
    const float fs = bw;
    const float kd = kdm_f() * dm;
    const float fhi = f0 + bw;
    const double lo = 1.0 / std::pow((double)f0, 2.0);
    const double hi = 1.0 / std::pow((double)fhi, 2.0);
    const float inv_fs = 1.0f / fs;
    const double v = std::floor((double)kd * (lo - hi) / (double)inv_fs);
    return v > 0.0 ? (unsigned long)v : 0ul;
}

unsigned long msosm_min_order(unsigned long Nd)
{
    if (Nd == 0)
        return 0;
    const double order = 2 * std::sqrt((double)Nd);
    return (unsigned long)std::pow(2.0, std::ceil(std::log2(order)));
}

unsigned long osm_min_order(unsigned long Nd)
{
    // int order = next_power_of_2((int)Nd); M = 2 * order
    int n = (int)Nd;
    int p;
    if (n <= 0) {
        p = 1;
    } else {
        unsigned int u = (unsigned int)(n - 1);
        u |= u >> 1;
        u |= u >> 2;
        u |= u >> 4;
        u |= u >> 8;
        u |= u >> 16;
        p = (int)(u + 1);
    }
    return 2ul * (unsigned long)p;
}

int delay_count(unsigned long Nd, unsigned long M)
{
    if (M == 0)
        return 0;
    return (int)std::ceil((float)Nd / (float)M);  // float quotient, ceil of a float
}

int segment_delays(float bw, float dm, float f0, unsigned long Nd, unsigned long M, int *delays)
{
    const unsigned long N = 2 * M;
    for (unsigned long k = 0; k < N; ++k)
        delays[k] = 0;
    const int dc = delay_count(Nd, M);
    if (dc <= 0)
        return 0;
    const float fs = bw;
    const float kdm = kdm_f();
    const float w0 = (float)(2 * kPi * f0);
    // Normalised segment edges in [-1, 1] (msosm_prepare.cpp:95-105): the
    // frequency whose delay behind the band bottom is j*M samples.
    std::vector<float> edge(dc + 1);
    edge[0] = -1.0f;
    edge[dc] = 1.0f;
    int first_pos = 1;
    const double inv_w02 = 1.0 / std::pow((double)w0, 2.0);
    const double c = 4 * kPi * kPi * (double)kdm * (double)dm;
    for (int j = 1; j < dc; ++j) {
        const float jm = (float)((unsigned long)j * M) / fs;  // float quotient
        const double s = std::sqrt(1.0 / (inv_w02 - (double)jm / c));
        edge[j] = (float)((s - (double)w0 - kPi * (double)fs) / kPi / (double)fs);
        if (edge[j] < 0)
            first_pos = j + 1;
    }
    const int negcount = first_pos;
    const int poscount = dc - first_pos + 1;
    // Negative frequencies occupy bins [M, 2M), positive [0, M)
    // (msosm_prepare.cpp:112-147); the segment straddling DC keeps one delay.
    for (int j = 0; j < negcount; ++j) {
        const unsigned long lo = (unsigned long)std::floor((edge[j] + 2.0f) * (float)M);
        const unsigned long hi = (j + 1 < negcount)
                                     ? (unsigned long)std::floor((edge[j + 1] + 2.0f) * (float)M)
                                     : N;
        for (unsigned long k = lo; k < hi && k < N; ++k)
            delays[k] = j;
    }
    unsigned long lo = 0;
    for (int j = 0; j < poscount; ++j) {
        const unsigned long hi = (unsigned long)std::floor(edge[j + negcount] * (float)M);
        for (unsigned long k = lo; k < hi && k < N; ++k)
            delays[k] = negcount - 1 + j;
        lo = hi;
    }
    return dc;
}

ChirpParams chirp_params(float bw, float dm, float f0, unsigned long M)
{
    ChirpParams p;
    p.fs = bw;
    p.kdm = kdm_f();
    p.dm = dm;
    p.w0 = (float)(2 * kPi * f0);
    p.step = (float)(2 * kPi * (double)bw / (double)M);
    return p;
}

// ---------------------------------------------------------------------------
// fold planner
// ---------------------------------------------------------------------------

FoldPlanner::FoldPlanner(float period, float fs, unsigned long discard_Nd, bool discard_set)
{
    // fold_gpu.cpp:3-8,29-33
    psf_ = period * fs;
    ps_ = (unsigned long)psf_;
    diff_ = psf_ - (float)ps_;
    discard_count_ = discard_set ? (int)std::ceil((float)discard_Nd / psf_) : 0;
    // Fold_GPU never sets its ready flag when the discard count is 0
    // (discard_samples not called, or Nd == 0): it folds nothing.  Here a
    // discard count of 0 means that nothing is discarded.
    if (discard_count_ == 0)
        ready_ = true;
}

void FoldPlanner::count_period()
{
    if (!ready_) {
        cur_discard_ += 1;
        if (cur_discard_ == discard_count_) {
            ready_ = true;
            cur_discard_ = 0;
        }
    }
}

void FoldPlanner::chunk(unsigned long size, std::vector<FoldSpan> &spans, bool &flush_pending)
{
    // Mirrors fold_gpu.cpp:48-173 with ranges in place of per-sample loops.
    // A skip that falls exactly at the chunk end wraps the reference's
    // unsigned counter; it is deferred to the next chunk, and in the
    // first branch (:98-109) the period is then not counted towards the
    // discard, as in the reference.
    spans.clear();
    flush_pending = false;
    const unsigned long ps = ps_;
    if (ps == 0)
        return;
    unsigned long cs = size, ci = 0;
    auto emit = [&](unsigned long a, unsigned long n, unsigned long phase0, bool completes, bool ready) {
        FoldSpan s;
        s.a = (int64_t)a;
        s.b = (int64_t)(a + n);
        s.phase0 = (int32_t)phase0;
        s.dest = ready ? (completes ? 1 : 2) : 0;
        s.period = period_no_;
        spans.push_back(s);
    };
    if (cur_diff_ > 1.0f) {
        cur_diff_ -= 1.0f;
        ci += 1;
        cs -= 1;
        if (cs == 0)
            return;
    }
    if (cur_idx_ != 0) {
        if (cs < ps - cur_idx_) {
            emit(ci, cs, cur_idx_, false, open_ready_);
            cur_idx_ += cs;
            return;
        }
        const unsigned long n = ps - cur_idx_;
        emit(ci, n, cur_idx_, true, open_ready_);
        if (open_ready_) {
            flush_pending = true;
            completed_ += 1;
        }
        cs -= n;
        ci += n;
        cur_idx_ = 0;
        period_no_ += 1;
        cur_diff_ += diff_;
        if (cur_diff_ > 1.0f) {
            cur_diff_ -= 1.0f;
            ci += 1;
            if (cs == 0) {
                cur_diff_ += 1.0f;
                return;
            }
            cs -= 1;
        }
        count_period();
    }
    while (cs >= ps) {
        emit(ci, ps, 0, true, ready_);
        if (ready_)
            completed_ += 1;
        cs -= ps;
        ci += ps;
        period_no_ += 1;
        cur_diff_ += diff_;
        bool wrap = false;
        if (cur_diff_ > 1.0f) {
            cur_diff_ -= 1.0f;
            ci += 1;
            if (cs == 0)
                wrap = true;
            else
                cs -= 1;
        }
        count_period();
        if (wrap) {
            cur_diff_ += 1.0f;
            return;
        }
    }
    if (cs > 0) {
        open_ready_ = ready_;
        emit(ci, cs, 0, false, ready_);
        cur_idx_ = cs;
    }
}

}  // namespace msosm
