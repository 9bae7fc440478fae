// sweep2_k2.cu -- schedule-3 sweep kernel instances for 2 words per lane
// (padded disparity count 128); one translation unit per width keeps the build parallel.
#include "sweep2_inst.cuh"

LUMEN_SWEEP2_INSTANCE(2)
