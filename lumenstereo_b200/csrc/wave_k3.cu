// wave_k3.cu -- schedule-4 wave kernel instances for padded disparity count 192;
// one translation unit per width keeps the build parallel.
#include "wave_inst.cuh"

LUMEN_WAVE_INSTANCE(3)
LUMEN_WAVE_TEAM_INSTANCE(3, 16)
