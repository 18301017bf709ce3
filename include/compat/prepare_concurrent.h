// prepare_concurrent.h -- include-name compatibility header for the reference's
// dedispersion/include/prepare_concurrent.h.  Its class (Prepare_MSOSM_DM_concurrent) is folded into
// MSOSM_GPU_DM_concurrent of the drop-in msosm_gpu_b200.hpp: the per-trial
// fields M, M_min, Nd, delaycount, dedisp_params and delay_points and the
// methods calculate_min_order, override_order, segmentation(i) and
// generate_dedisp_params(i) are members of that class.
#pragma once

#include "globals.h"
