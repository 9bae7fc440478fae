// sweep2_k8.cu -- schedule-3 sweep kernel instances for 8 words per lane
// (padded disparity count 512); one translation unit per width keeps the build parallel.
#include "sweep2_inst.cuh"

LUMEN_SWEEP2_INSTANCE(8)
