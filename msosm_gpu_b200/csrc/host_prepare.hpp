// host_prepare.hpp -- host-side filter-design arithmetic and the fold planner.
//
// The integer results here (Nd, minimum orders, delaycount, per-bin delays,
// which output samples fold into which phase bin) must equal the reference's
// bit for bit, so each function reproduces the reference's float/double
// promotion sequence step by step (cited per function).  Compiled with
// -ffp-contract=off: a fused multiply-add would change these integers.
#pragma once

#include <cstdint>
#include <vector>

namespace msosm {

// Reference constants: `constexpr auto pi = M_PI` (utils/include/globals.h:29)
// and `kdm = 4.15 * 1e15` stored in a float (msosm_prepare.cpp:6).
constexpr double kPi = 3.14159265358979323846;
inline float kdm_f() { return (float)(4.15 * 1e15); }

// msosm_prepare.cpp:3-8 (Nd); 0 for dm <= 0.
unsigned long dispersion_smear(float bw, float dm, float f0);
// msosm_prepare.cpp:17-24
unsigned long msosm_min_order(unsigned long Nd);
// osm_prepare.cpp:17-30,86-99
unsigned long osm_min_order(unsigned long Nd);
// msosm_prepare.cpp:88
int delay_count(unsigned long Nd, unsigned long M);
// msosm_prepare.cpp:86-152; fills delays[2M], returns delaycount.
int segment_delays(float bw, float dm, float f0, unsigned long Nd, unsigned long M, int *delays);

// Parameters of the chirp h of msosm_prepare.cpp:40-63 for the device design
// kernel: the float-rounded quantities the reference computes once.
struct ChirpParams {
    float fs, kdm, dm, w0, step;
};
ChirpParams chirp_params(float bw, float dm, float f0, unsigned long M);

// One run of consecutive output samples of one fold period inside a chunk.
struct FoldSpan {
    int64_t a, b;     // chunk-local sample range [a, b)
    int32_t phase0;   // phase of sample a within its period
    int32_t dest;     // 0: not folded, 1: fold now (period completes in this chunk),
                      // 2: fold into the pending accumulator (period still open)
    int64_t period;   // global period index
};

// Dry run of the Fold_GPU state machine (folding/fold_gpu.cpp:48-173) on
// sample counts only.  Successive chunk() calls continue one stream.
class FoldPlanner {
public:
    FoldPlanner(float period, float fs, unsigned long discard_Nd, bool discard_set);
    // Spans of one chunk of `size` output samples, in sample order.
    // flush_pending is set when the period left open by the previous chunk is
    // folded and completes in this one: its earlier samples must move from
    // the pending accumulator into the profile before this chunk is folded.
    void chunk(unsigned long size, std::vector<FoldSpan> &spans, bool &flush_pending);
    unsigned long period_samples() const { return ps_; }
    unsigned long long completed_folded() const { return completed_; }

private:
    void count_period();
    unsigned long ps_ = 0;
    float psf_ = 0.f, diff_ = 0.f, cur_diff_ = 0.f;
    unsigned long cur_idx_ = 0;
    bool ready_ = false;
    int discard_count_ = 0, cur_discard_ = 0;
    int64_t period_no_ = 0;
    bool open_ready_ = false;  // the open (incomplete) period was processed while ready
    unsigned long long completed_ = 0;
};

}  // namespace msosm
