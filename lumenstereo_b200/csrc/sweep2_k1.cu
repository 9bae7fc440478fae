// sweep2_k1.cu -- schedule-3 sweep kernel instances for 1 words per lane
// (padded disparity count 64); one translation unit per width keeps the build parallel.
#include "sweep2_inst.cuh"

LUMEN_SWEEP2_INSTANCE(1)
