// sweep2_k7.cu -- schedule-3 sweep kernel instances for 7 words per lane
// (padded disparity count 448); one translation unit per width keeps the build parallel.
#include "sweep2_inst.cuh"

LUMEN_SWEEP2_INSTANCE(7)
