// wave_k4.cu -- schedule-4 wave kernel instances for padded disparity count 256;
// one translation unit per width keeps the build parallel.
#include "wave_inst.cuh"

LUMEN_WAVE_INSTANCE(4)
LUMEN_WAVE_TEAM_INSTANCE(4, 16)
