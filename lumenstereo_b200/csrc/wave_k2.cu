// wave_k2.cu -- schedule-4 wave kernel instances for padded disparity count 128;
// one translation unit per width keeps the build parallel.
#include "wave_inst.cuh"

LUMEN_WAVE_INSTANCE(2)
LUMEN_WAVE_TEAM_INSTANCE(2, 8)
LUMEN_WAVE_TEAM_INSTANCE(2, 16)
