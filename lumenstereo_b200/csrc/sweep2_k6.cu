// sweep2_k6.cu -- schedule-3 sweep kernel instances for 6 words per lane
// (padded disparity count 384); one translation unit per width keeps the build parallel.
#include "sweep2_inst.cuh"

LUMEN_SWEEP2_INSTANCE(6)
