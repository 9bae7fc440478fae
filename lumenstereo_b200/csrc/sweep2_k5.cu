// sweep2_k5.cu -- schedule-3 sweep kernel instances for 5 words per lane
// (padded disparity count 320); one translation unit per width keeps the build parallel.
#include "sweep2_inst.cuh"

LUMEN_SWEEP2_INSTANCE(5)
