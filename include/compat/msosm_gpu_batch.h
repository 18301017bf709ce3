// msosm_gpu_batch.h -- include-name compatibility header for the reference's
// dedispersion/include/msosm_gpu_batch.h: the classes it declared, from the drop-in msosm_gpu_b200.hpp
// (they run on libmsosm_b200.so), in the global namespace where the
// reference's drivers look for them.
#pragma once

#include "globals.h"

using msosm_b200::Prepare_MSOSM;
using msosm_b200::MSOSM_GPU_BATCH;
using msosm_b200::MSOSM_GPU_DM_BATCH_loop;
