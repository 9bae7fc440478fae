// sweep2_k3.cu -- schedule-3 sweep kernel instances for 3 words per lane
// (padded disparity count 192); one translation unit per width keeps the build parallel.
#include "sweep2_inst.cuh"

LUMEN_SWEEP2_INSTANCE(3)
