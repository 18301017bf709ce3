// Fold_GPU's raw-resolution fields through the drop-in header: fold_count
// and tmp_fold (folding/include/fold_gpu.h:27-28) with track_raw_state, and
// the per-trial prepare fields of MSOSM_GPU_DM_concurrent
// (dedispersion/include/prepare_concurrent.h:10-38).  Prints them for the
// test to check.
#include <cstdio>
#include <vector>

#include "msosm_gpu_b200.hpp"

using namespace msosm_b200;

int main()
{
    // 100 samples per period exactly (0.25 s at 400 Hz), no drift, chunks of
    // 64 samples: 10 chunks = 6 complete periods + 40 samples of the 7th
    const unsigned long size = 64;
    Fold_GPU fold(0.25f, 400.f, size, "/dev/null", 10);
    fold.track_raw_state = true;
    for (int c = 0; c < 10; ++c) {
        for (unsigned long i = 0; i < size; ++i) {
            const unsigned long t = c * size + i;
            fold.total_intensity[i] = (t % 7 == 0) ? 0.f : (float)(1 + t);
        }
        fold.load_total_intensity();
        fold.fold_data();
    }
    std::printf("period_samples %lu\n", fold.period_samples);
    std::printf("fold_count");
    for (unsigned long p = 0; p < fold.period_samples; ++p)
        std::printf(" %lu", fold.fold_count[p]);
    std::printf("\ntmp_fold");
    for (unsigned long p = 0; p < 40; ++p)
        std::printf(" %.0f", fold.tmp_fold[p]);
    std::printf("\n");

    float bw[3] = {16e6f, 16e6f, 16e6f}, dm[3] = {10.f, 50.f, 73.2f}, f0[3] = {1242e6f, 1242e6f, 1242e6f};
    MSOSM_GPU_DM_concurrent m(bw, dm, f0, 3);
    m.calculate_min_order();
    std::printf("M_min %lu %lu %lu common %lu\n", m.M_min[0], m.M_min[1], m.M_min[2], m.M_common_min);
    m.override_order(2048);
    for (int i = 0; i < 3; ++i) {
        m.segmentation(i);
        m.generate_dedisp_params(i);
    }
    std::printf("prepared delaycount %d %d %d d[100] %d H[7] %.9g %.9g\n", m.delaycount[0], m.delaycount[1],
                m.delaycount[2], m.delay_points[2][100], m.dedisp_params[2][7].x, m.dedisp_params[2][7].y);
    m.initialize_uint16(4096, 2);
    std::printf("handle delaycount %d %d %d d[100] %d H[7] %.9g %.9g M %lu %lu %lu Nd %lu\n", m.delaycount[0],
                m.delaycount[1], m.delaycount[2], m.delay_points[2][100], m.dedisp_params[2][7].x,
                m.dedisp_params[2][7].y, m.M[0], m.M[1], m.M[2], m.Nd[2]);
    return 0;
}
