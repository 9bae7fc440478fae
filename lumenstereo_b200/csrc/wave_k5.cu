// wave_k5.cu -- schedule-4 wave kernel instances for padded disparity count 320;
// one translation unit per width keeps the build parallel.
#include "wave_inst.cuh"

LUMEN_WAVE_INSTANCE(5)
LUMEN_WAVE_TEAM_INSTANCE(5, 16)
