// sweep2_k4.cu -- schedule-3 sweep kernel instances for 4 words per lane
// (padded disparity count 256); one translation unit per width keeps the build parallel.
#include "sweep2_inst.cuh"

LUMEN_SWEEP2_INSTANCE(4)
