// wave_k1.cu -- schedule-4 wave kernel instances for padded disparity count 64;
// one translation unit per width keeps the build parallel.
#include "wave_inst.cuh"

LUMEN_WAVE_INSTANCE(1)
LUMEN_WAVE_TEAM_INSTANCE(1, 8)
LUMEN_WAVE_TEAM_INSTANCE(1, 16)
